"""The C ABI library loads and exports exactly what include/orihime_b200.h declares (CPU)."""

import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "orihime_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(swb_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from orihime_b200 import _lib

    return _lib.load()


def test_header_declares_entry_points():
    names = _declared()
    assert "swb_sw_affine_forward" in names and "swb_sw_forward" in names
    assert len(names) >= 7


def test_library_exports_every_declared_symbol(lib):
    from orihime_b200 import _lib

    out = subprocess.run(["nm", "-D", "--defined-only", _lib.path()], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (swb_[a-z0-9_]+)", out))
    missing = [n for n in _declared() if n not in exported]
    assert not missing, missing
    for n in _declared():
        assert hasattr(lib, n)


def test_abi_version_and_errors(lib):
    assert lib.swb_abi_version() == 2
    assert lib.swb_error_string(0) == b"ok"
    assert b"workspace" in lib.swb_error_string(-2)


def test_workspace_sizes_monotone(lib):
    a = lib.swb_sw_affine_workspace_bytes(4, 100, 100)
    b = lib.swb_sw_affine_workspace_bytes(8, 100, 100)
    c = lib.swb_sw_affine_workspace_bytes(4, 200, 300)
    assert 0 < a < b and a < c
    assert lib.swb_sw_affine_workspace_bytes(0, 10, 10) == 0
    assert 0 < lib.swb_sw_workspace_bytes(4, 100, 100) < a
    # checkpoints every 4 wavefront steps: at most 2.25 floats per cell (2 columns
    # per lane; 1.875 at 4) plus the cross-band buffers, below the 3 floats per
    # cell of one fp32 three-state table (the reference keeps alpha and beta)
    full = 3 * 4 * 16385 * 16385 * 4
    assert lib.swb_sw_affine_workspace_bytes(4, 16384, 16384) < 0.85 * full


def test_argument_errors_return_before_any_launch(lib):
    # these return before touching CUDA, so they run on a CPU-only host too
    f = ctypes.c_float
    rc = lib.swb_sw_affine_forward(None, None, 1, 4, 4, f(-2), f(-0.5), f(0.0), None, None, None,
                                   None, None, None, 0, None, None)
    assert rc == -1  # temperature must be > 0
    rc = lib.swb_sw_affine_forward(None, None, -1, 4, 4, f(-2), f(-0.5), f(1.0), None, None, None,
                                   None, None, None, 0, None, None)
    assert rc == -1
    rc = lib.swb_sw_forward(None, None, 0, 4, 4, f(-1), f(1.0), None, None, None, None, None, 0,
                            None, None)
    assert rc == 0  # empty batch: nothing to do
    buf = (ctypes.c_float * 16)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    rc = lib.swb_sw_affine_forward(p, None, 1, 4, 4, f(-2), f(-0.5), f(1.0), p, p, p, p, p, p, 16,
                                   None, None)
    assert rc == -2  # workspace too small


@pytest.mark.parametrize("fam", ["nw", "nw_affine", "sv_affine"])
def test_other_families_argument_errors_and_workspaces(lib, fam):
    """The global and Saigo-Vert entry points validate like the local ones,
    before touching CUDA: temperature <= 0 and B < 0 are argument errors, an
    empty batch is a no-op, a short workspace is refused."""
    f = ctypes.c_float
    ws = getattr(lib, f"swb_{fam}_workspace_bytes")
    a, b = ws(4, 100, 100), ws(8, 100, 100)
    assert 0 < a < b and ws(0, 10, 10) == 0
    assert getattr(lib, f"swb_{fam}_value_workspace_bytes")(4, 100, 100) > 0
    assert getattr(lib, f"swb_{fam}_aux_workspace_bytes")(4, 100, 100) > 0
    fwd = getattr(lib, f"swb_{fam}_forward")
    buf = (ctypes.c_float * 16)()
    p = ctypes.cast(buf, ctypes.c_void_p)
    if fam == "nw":
        call = lambda B, T, w, n: fwd(w, None, B, 4, 4, f(-1), f(T), w, w, w, w, w, n, None, None)  # noqa: E731
    else:
        call = lambda B, T, w, n: fwd(w, None, B, 4, 4, f(-2), f(-0.5), f(T), w, w, w, w, w, w, n,  # noqa: E731
                                      None, None)
    assert call(1, 0.0, None, 0) == -1
    assert call(-1, 1.0, None, 0) == -1
    assert call(0, 1.0, None, 0) == 0
    assert call(1, 1.0, p, 16) == -2


@pytest.mark.parametrize("fam", ["sw_affine", "sw"])
def test_aux_workspace_for_parameters(lib, fam):
    """Second-order workspace sizes (host arithmetic only): with every gap <= 0
    and 0 < T < inf the linear-domain tangent kernels run, and their
    checkpoints need a small fraction of the log-domain field table that the
    any-parameters size covers; other parameters get that table's size."""
    f = ctypes.c_float
    any_ = getattr(lib, f"swb_{fam}_aux_workspace_bytes")
    for_ = getattr(lib, f"swb_{fam}_aux_workspace_bytes_for")
    gaps = (f(-2.0), f(-0.5)) if fam == "sw_affine" else (f(-1.0),)
    pos = (f(-2.0), f(0.25)) if fam == "sw_affine" else (f(0.25),)
    B, L1, L2 = 256, 512, 512
    n_any = int(any_(B, L1, L2))
    n_lin = int(for_(B, L1, L2, *gaps, f(0.5)))
    assert 0 < n_lin * 8 < n_any
    assert int(for_(B, L1, L2, *pos, f(0.5))) == n_any          # a positive gap: log domain
    assert int(for_(B, L1, L2, *gaps, f(0.0))) == n_any         # T <= 0: no tangent kernels
    assert int(for_(0, L1, L2, *gaps, f(0.5))) == 0
    assert int(for_(2 * B, L1, L2, *gaps, f(0.5))) > n_lin


@pytest.mark.parametrize("fam,params", [("sw_affine", (-2.0, -0.5, 0.5)), ("sw", (-1.0, 0.5)),
                                        ("sw_affine", (-2.0, 0.25, 0.5)), ("nw_affine", (-2.0, -0.5, 0.5)),
                                        ("sv_affine", (-2.0, -0.5, 0.5))])
def test_second_order_pair_groups(monkeypatch, fam, params):
    """The op layer's pair-group plan for second-order calls (host logic):
    under stream capture there is no free-memory query and the budget is the
    2 GiB floor.  Groups then fit the budget, cover the batch, and the
    workspace fits every group; the local models with every gap <= 0 are
    sized for their tangent kernels (far fewer groups), the others for the
    log-domain field table."""
    from orihime_b200 import _ops

    monkeypatch.setattr(_ops, "_capturing", lambda: True)
    B, L = 4096, 512
    g, nbytes = _ops._aux_plan(fam, B, L, L, None, params)
    if fam in _ops._AUX_FOR:
        size = lambda b: int(getattr(_ops._LIB, _ops._AUX_FOR[fam])(b, L, L, *map(float, params)))  # noqa: E731
    else:
        size = lambda b: int(getattr(_ops._LIB, _ops._AUX[fam][0])(b, L, L))  # noqa: E731
    budget = 2 << 30
    assert 1 <= g <= B and nbytes <= budget
    groups = list(_ops._groups(B, g))
    assert groups[0][0] == 0 and groups[-1][1] == B
    assert all(b1 > b0 and b1 - b0 <= g for b0, b1 in groups)
    assert all(groups[k][1] == groups[k + 1][0] for k in range(len(groups) - 1))
    assert all(size(b1 - b0) <= nbytes for b0, b1 in groups)
    if fam in ("sw_affine", "sw") and all(p <= 0 for p in params[:-1]):
        assert len(groups) <= 5            # about 7 B per cell: 8.4 GB affine
    else:
        assert len(groups) >= 40           # about 100 B per cell: 92 GB affine
    # a batch within the budget is one group
    g1, n1 = _ops._aux_plan(fam, 8, L, L, None, params)
    assert g1 == 8 and n1 == size(8)
