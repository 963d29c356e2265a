"""One rank of the two-process CPU test of the multi-process plumbing
(launched by tests/test_dist.py through torch.distributed.run, gloo).

Each rank steps its own block of rows of the 64 x 64 4,096-cell random field with the
oracle and writes its block; rank 0 also records the max-over-ranks value."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main(out_dir: str) -> int:
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
    o = m.chem_step(f.dt, f.T[sel], f.rho[sel], f.Y[:, sel], threads=1)
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), o["Y_prod"])
    mx = dist.max_over_ranks(float(rank + 1))
    dist.barrier()
    if rank == 0:
        with open(os.path.join(out_dir, "max.txt"), "w") as fh:
            fh.write(repr(mx))
    tdist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1]))
