"""torch.autograd wrapper of the Pi forward/backward pair (test harness only).

PiFunction.apply(mu, kappa, gauge) -> Pi (real tensor, 32*V: re/im pairs in
the conn layout).  Its backward calls cvcb_pi_backward with the incoming
gradient as weights: for a real L, dL/dPi given as real pairs (g_re, g_im)
is exactly L = Re sum conj(g) Pi to first order.
"""
import numpy as np
import torch


class PiFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mu, kappa, gauge, lat, source_site, params):
        lat.set_params(float(kappa), float(mu), lat.BCangle)
        lat.upload_gauge(gauge.detach().cpu().numpy())
        conn, _ = lat.pi_forward(source_site, params)
        ctx.lat = lat
        return torch.from_numpy(conn.copy())

    @staticmethod
    def backward(ctx, grad_conn):
        w = grad_conn.detach().cpu().numpy().astype(np.float64)
        dmu, dka, gu = ctx.lat.pi_backward(w)
        return (torch.tensor(dmu, dtype=torch.float64), torch.tensor(dka, dtype=torch.float64),
                torch.from_numpy(gu), None, None, None)
