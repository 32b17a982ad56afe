"""fiim_prec_apply_noalloc: the preconditioner product for callers that cannot allocate
device memory when they call (their memory belongs to a pool set up at start-up, or to a
fixed per-process budget). It keeps its intermediate vector in a fixed array inside the
library instead of caller scratch.

Checked through the C-ABI against fiim_prec_apply, which the other GPU tests pin to the
oracle: the two must agree bit for bit (the tolerance the preconditioner tests use), on two
calls in a row, so a call cannot lean on what the previous one left in the shared array.
This file is collected last; it passes alone in a fresh process and after the others.
"""
import ctypes as C

import numpy as np
import pytest

import fiim_b200 as FB
from conftest import sub

pytestmark = pytest.mark.gpu


def _t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _factors(g, prefix, dev):
    F = sub(g, prefix)
    return F, {k: _t(F[k], dev) for k in ("Gi", "Gj", "Gv", "IDv", "Hi", "Hj", "Hv")}


def _both(d, r, n, dev):
    import torch
    z_ref = torch.full((n,), np.nan, dtype=torch.float64, device=dev)
    z_na = torch.full((n,), np.nan, dtype=torch.float64, device=dev)
    tm = torch.empty(n, dtype=torch.float64, device=dev)
    FB.prec_apply(d["Gi"], d["Gj"], d["Gv"], d["IDv"], d["Hi"], d["Hj"], d["Hv"], r, z_ref, tm)
    FB.prec_apply_noalloc(d["Gi"], d["Gj"], d["Gv"], d["IDv"], d["Hi"], d["Hj"], d["Hv"], r, z_na)
    torch.cuda.synchronize()
    return z_ref.cpu().numpy(), z_na.cpu().numpy()


def test_noalloc_matches_prec_apply_on_consecutive_calls(golden, cuda):
    # A larger system, then a smaller one: the second call reads only what it wrote itself.
    for name, prefix in (("poisson128_afiim", ""), ("convdiff16_pdfiim", ""), ("poisson128_afiim", "")):
        g = golden(name)
        F, d = _factors(g, prefix, cuda)
        n = len(g["b"])
        for seed in (1, 2):
            r = _t(FB.rand_normal(n, seed), cuda)
            z_ref, z_na = _both(d, r, n, cuda)
            assert np.isfinite(z_na).all()
            assert np.array_equal(z_na, z_ref)
        assert np.array_equal(_both(d, _t(F["u"], cuda), n, cuda)[1], F["Mu"])


def test_noalloc_rejects_systems_beyond_its_limit(cuda):
    import torch
    n = (1 << 20) + 1
    i = torch.zeros(n + 1, dtype=torch.int32, device=cuda)
    v = torch.zeros(1, dtype=torch.float64, device=cuda)
    x = torch.zeros(n, dtype=torch.float64, device=cuda)
    rc = FB.lib().fiim_prec_apply_noalloc(C.c_int(n), *[FB._ptr(a) for a in (i, i, v, x, i, i, v, x, x)], None)
    assert rc == FB.FIIM_EARG
    assert "1048576" in FB.lib().fiim_last_error().decode()
