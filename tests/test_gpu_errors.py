"""The error paths of the C ABI, made to happen without a GPU fault.

- GLIDE_ERR_NONFINITE: a NaN placed in the thickness on the host makes the
  first residual norm non-finite, and glide_forward returns the code.
- GLIDE_ERR_TIMEOUT: the tuning switch GLIDE_TUNE_TMA_GIVE_UP makes every
  stencil block's first wait for its staged tile copies give up at once.  The
  block still waits (bounded) for the copies to land, then returns; the host
  finds the error word at the next norm read.  Nothing waits without a limit.

After either error the same handle, with its inputs restored, solves cleanly
and matches the reference's C1 forward fixture (1e-10), so an error leaves
the handle usable.
"""
from __future__ import annotations

import numpy as np
import pytest

from util import load_golden, rel_err

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DT = 10.0


def _c1_handle():
    from glide_b200.hierarchy import Hierarchy
    g = load_golden("c1_forward_f64")
    h = Hierarchy(64, 64, 1000.0, 4, precision="fp64")
    return h, g


def _load(h, g):
    for k in ("bed", "B", "beta", "smb", "H", "H_prev"):
        h.set(k, 0, torch.as_tensor(g[f"in_{k}"]), restrict_down=True)
    for k in ("u", "v", "mask"):
        h.set(k, 0, 0.0, restrict_down=True)


def _check_clean_solve(h, g):
    _load(h, g)
    h.set_fas(False, maximum_vcycles=3, relative_tolerance=0.0, absolute_tolerance=0.0)
    st = h.forward(DT, 0)
    assert st["vcycles"] == 3
    for k in ("u", "v", "H"):
        assert rel_err(h.view(k, 0).cpu().numpy(), g[f"out_{k}"]) <= 1e-10, k


def test_nan_thickness_returns_nonfinite():
    from glide_b200 import _lib
    h, g = _c1_handle()
    _load(h, g)
    H = torch.as_tensor(g["in_H"]).clone()
    H[17, 23] = float("nan")
    h.set("H", 0, H, restrict_down=True)
    h.set_fas(False, maximum_vcycles=3, relative_tolerance=0.0, absolute_tolerance=0.0)
    with pytest.raises(_lib.GlideError) as e:
        h.forward(DT, 0)
    assert e.value.code == _lib.GLIDE_ERR_NONFINITE
    assert "not finite" in str(e.value)
    _check_clean_solve(h, g)


@pytest.mark.parametrize("graphs", [True, False])
def test_tile_wait_give_up_returns_timeout(graphs):
    from glide_b200 import _lib
    h, g = _c1_handle()
    h.set_use_graphs(graphs)
    _load(h, g)
    h.set_fas(False, maximum_vcycles=3, relative_tolerance=0.0, absolute_tolerance=0.0)
    h.set_tuning(tma_give_up=True)
    with pytest.raises(_lib.GlideError) as e:
        h.forward(DT, 0)
    assert e.value.code == _lib.GLIDE_ERR_TIMEOUT
    # a residual alone reports it too
    with pytest.raises(_lib.GlideError) as e:
        h.residual(0, DT, _lib.USE_MASK, norms=True)
    assert e.value.code == _lib.GLIDE_ERR_TIMEOUT
    torch.cuda.synchronize()  # the context is intact
    h.set_tuning(tma_give_up=False)
    _check_clean_solve(h, g)
    assert np.isfinite(h.residual(0, DT, _lib.USE_MASK, norms=True)).all()
