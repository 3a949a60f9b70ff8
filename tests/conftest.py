"""Shared test configuration.

Markers: ``gpu`` -- needs a CUDA device (run with ``-m gpu``); everything else runs on CPU.

Tolerances (also stated in each test that uses them):
  * forward vs the reference CUDA kernels:  per element |d| <= 1e-5 |ref| + 1e-5 * 1e-3 * max|ref|
    (the shading sums are sums of non-negative terms, so relative error is meaningful down to
    the tiny floor);
  * gradients vs the reference:  per tensor max|d| / max|ref| <= 1e-4 and per element
    |d| <= 1e-4 |ref| + 1e-4 * 0.1 * max|ref| (gradients cancel, so elements far below the
    tensor's scale are held to an absolute floor tied to that scale);
  * against the FP64 oracle the same bounds apply; the env-map gradient is compared against
    the FP64 oracle with the gradient bound.
"""
import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")

FWD_RTOL = 1e-5
FWD_FLOOR = 1e-3
GRAD_RTOL = 1e-4
GRAD_FLOOR = 0.1


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _np(x):
    if hasattr(x, "detach"):
        x = x.detach().cpu().numpy()
    return np.asarray(x, dtype=np.float64)


def err_stats(got, ref):
    """(max |d| / max |ref|, max over elements of |d| / (|ref| + floor*max|ref|)) for FWD floor."""
    g, r = _np(got), _np(ref)
    scale = max(np.abs(r).max(), 1e-30) if r.size else 1.0
    d = np.abs(g - r)
    return float(d.max() / scale) if d.size else 0.0, d, scale


def assert_close_fwd(got, ref, name="", rtol=FWD_RTOL, floor=FWD_FLOOR, allowance=None):
    """Per element |got - ref| <= rtol (|ref| + floor max|ref|) + allowance (an optional per-element
    array: the reference's own measured deviation from exact arithmetic)."""
    g, r = _np(got), _np(ref)
    assert g.shape == r.shape, (name, g.shape, r.shape)
    if r.size == 0:
        return
    assert np.isfinite(g).all(), f"{name}: non-finite values"
    scale = max(np.abs(r).max(), 1e-30)
    bound = rtol * np.abs(r) + rtol * floor * scale
    if allowance is not None:
        bound = bound + _np(allowance)
    d = np.abs(g - r)
    worst = np.argmax(d - bound)
    assert (d <= bound).all(), (f"{name}: max rel err {np.max(d / (np.abs(r) + floor * scale)):.3e} "
                                f"at {np.unravel_index(worst, d.shape)} got {g.flat[worst]!r} ref {r.flat[worst]!r}")


def assert_close_grad(got, ref, name="", rtol=GRAD_RTOL, floor=GRAD_FLOOR, allowance=None):
    """Per tensor max|got - ref| / max|ref| <= rtol and per element
    |got - ref| <= rtol (|ref| + floor max|ref|), both widened by an optional per-element allowance."""
    g, r = _np(got), _np(ref)
    assert g.shape == r.shape, (name, g.shape, r.shape)
    if r.size == 0:
        return
    assert np.isfinite(g).all(), f"{name}: non-finite values"
    scale = np.abs(r).max()
    if scale == 0:
        assert np.abs(g).max() == 0, f"{name}: expected zeros"
        return
    allow = np.zeros_like(r) if allowance is None else _np(allowance)
    d = np.abs(g - r)
    assert (d - allow).max() / scale <= rtol, f"{name}: tensor rel err {d.max() / scale:.3e}"
    bound = rtol * np.abs(r) + rtol * floor * scale + allow
    worst = np.argmax(d - bound)
    assert (d <= bound).all(), (f"{name}: element err {d.flat[worst]:.3e} vs bound {bound.flat[worst]:.3e} "
                                f"(ref {r.flat[worst]!r})")


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def reference_ext():
    """The reference extension built from its sources (oracle/_ref); skipped when absent."""
    refdir = os.path.join(ROOT, "oracle", "_ref")
    if not glob.glob(os.path.join(refdir, "_diff_envshade*.so")):
        pytest.skip("reference extension not built (python oracle/build_ref.py)")
    if refdir not in sys.path:
        sys.path.insert(0, refdir)
    import _diff_envshade
    return _diff_envshade


def golden_files(pattern="*.npz"):
    """Fixture files matching pattern; the etc_*.npz fixtures of the mesh and env-map helpers are
    listed only when the pattern names them."""
    files = sorted(glob.glob(os.path.join(GOLDEN, pattern)))
    if not pattern.startswith("etc_"):
        files = [f for f in files if not os.path.basename(f).startswith("etc_")]
    return files
