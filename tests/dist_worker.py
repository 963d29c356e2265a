"""One rank of the two-process CPU test of the multi-process plumbing
(launched by tests/test_dist.py through torch.distributed.run, gloo).

Each rank steps its own block of rows of the 64 x 64 4,096-cell random field
and writes its block; rank 0 also records the max-over-ranks value.  The
stepper is the oracle (CPU test of the plumbing) or, with "product" as the
second argument, the library's nrg_chem_step_device on cuda:0 (both ranks
share the one GPU; their kernels never wait on each other)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main(out_dir: str, stepper: str = "oracle") -> int:
    import torch.distributed as tdist
    from nrg_b200 import dist, fields, keromnes_paths
    from oracle import oracle_py as op
    rank, world, _ = dist.world()
    dist.init("gloo", timeout_s=120)
    m = op.Mechanism(*keromnes_paths(), 1.0, "cal.mol")
    f = fields.random_field(m.tables()["molar_mass"])
    side = f.shape[0]
    r0, r1 = dist.row_block(side, rank, world)
    sel = np.arange(r0 * side, r1 * side)
    if stepper == "product":
        Y_prod = step_rows_on_gpu(f, sel)
    else:
        Y_prod = m.chem_step(f.dt, f.T[sel], f.rho[sel], f.Y[:, sel], threads=1)["Y_prod"]
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), Y_prod)
    mx = dist.max_over_ranks(float(rank + 1))
    dist.barrier()
    if rank == 0:
        with open(os.path.join(out_dir, "max.txt"), "w") as fh:
            fh.write(repr(mx))
    tdist.destroy_process_group()
    return 0


def step_rows_on_gpu(f, sel):
    """This rank's cells through the product's device entry point."""
    import torch
    from nrg_b200 import keromnes_paths
    from nrg_b200.chemistry import ChemicalKineticsSolver
    dev = torch.device("cuda:0")
    T = torch.tensor(f.T[sel], device=dev)
    rho = torch.tensor(f.rho[sel], device=dev)
    Y = torch.tensor(np.ascontiguousarray(f.Y[:, sel]), device=dev)
    Yp, Yp2, Ef = torch.zeros_like(Y), torch.zeros_like(Y), torch.zeros_like(T)
    s = ChemicalKineticsSolver(None, *keromnes_paths(), mode="fast")
    try:
        s.step_device(f.dt, T, rho, Y, Yp, Yp2, Ef)
        torch.cuda.synchronize()
        return Yp.cpu().numpy()
    finally:
        s.close()


if __name__ == "__main__":
    sys.exit(main(*sys.argv[1:3]))
