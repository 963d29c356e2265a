"""Helpers shared by the GPU tests: run the product on torch CUDA tensors."""
import numpy as np


def to_dev(f):
    import torch
    dev = torch.device("cuda:0")
    return (torch.tensor(f.T, device=dev), torch.tensor(f.rho, device=dev), torch.tensor(f.Y, device=dev))


def run_device(solver, f, mode, bc=None, launch=None, graph=True, y_prod2_init=None):
    import torch
    T, rho, Y = to_dev(f)
    n = f.n
    Yp = torch.zeros_like(Y)
    Yp2 = torch.zeros_like(Y) if y_prod2_init is None else torch.tensor(y_prod2_init, device=Y.device)
    Ef = torch.zeros_like(T)
    Ta = torch.zeros_like(T)
    st = torch.zeros(n, dtype=torch.uint8, device=Y.device)
    bct = None if bc is None else torch.tensor(bc, dtype=torch.int8, device=Y.device)
    solver.set_mode(mode)
    solver.set_graph(graph)
    if launch is not None:
        solver.set_launch(**launch)
    stats = solver.step_device(f.dt, T, rho, Y, Yp, Yp2, Ef, bc=bct, T_after=Ta, status=st)
    torch.cuda.synchronize()
    return dict(Y_prod=Yp.cpu().numpy(), Y_prod2=Yp2.cpu().numpy(), E_f_prod=Ef.cpu().numpy(),
                T_after=Ta.cpu().numpy(), status=st.cpu().numpy()), stats


def dY(out, f):
    return out["Y_prod"] * f.dt / f.rho[None, :]
