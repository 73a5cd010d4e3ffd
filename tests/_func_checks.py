"""torch.func checks of the public functions (map, value, entropy), shared
by the CPU run (oracle-backed kernels, tests/_oracle_cpu_ops.py) and the GPU
run of tests/test_func_transforms.py.

They restate the reference's transform contract (tests/test_func_compat.py of
megure-labs/orihime): jvp, vjp, jacrev and vmap agree with eager autograd and
with central differences on [2, 3, 3] inputs with tensor parameters; eager
backward agrees with central differences; a mapped scalar parameter raises
the native ops' guard; forward mode under vmap (jacfwd) raises
NotImplementedError naming the jvp function; entropy's parameter directions
raise NotImplementedError.
"""

from __future__ import annotations

import torch

import orihime_b200 as ohm

# (public name, parameters (public name, value), raw parameter names)
CASES = {
    "sw": ((("gap_score", -0.7), ("temperature", 0.9)), ("gap", "temp")),
    "sw_affine": ((("gap_open_score", -1.0), ("gap_extend_score", -0.3), ("temperature", 0.9)),
                  ("gap_open", "gap_ext", "temp")),
    "nw": ((("gap_score", -0.7), ("temperature", 0.9)), ("gap", "temp")),
    "nw_affine": ((("gap_open_score", -1.0), ("gap_extend_score", -0.3), ("temperature", 0.9)),
                  ("gap_open", "gap_ext", "temp")),
    "sv_linear": ((("gap_score", -0.7), ("temperature", 0.9)), ("gap", "temp")),
    "sv_affine": ((("gap_open_score", -1.0), ("gap_extend_score", -0.3), ("temperature", 0.9)),
                  ("gap_open", "gap_ext", "temp")),
}
OBSERVABLES = ("map", "value", "entropy")
EPS = 1e-2


def target(name: str, observable: str):
    return getattr(ohm, name if observable == "map" else f"{name}_{observable}")


def scores(name: str, device, batch: int = 2, seed: int = 0) -> torch.Tensor:
    g = torch.Generator(device="cpu").manual_seed(5100 + seed + list(CASES).index(name))
    return (0.2 * torch.randn(batch, 3, 3, generator=g)).to(device)


def function_and_primals(name: str, observable: str, device):
    """f(primary[, params...]) and its primals; entropy takes the primary only."""
    params, _ = CASES[name]
    fn = target(name, observable)
    x = scores(name, device)
    if observable == "entropy":
        kw = dict(params)
        return (lambda p: fn(p, **kw)), (x,)
    names = [n for n, _ in params]
    prim = (x, *(torch.tensor(v, device=device) for _, v in params))
    return (lambda p, *ps: fn(p, **dict(zip(names, ps)))), prim


def _close(a, b, rtol=1e-4, atol=1e-5):
    a = a if isinstance(a, tuple) else (a,)
    b = b if isinstance(b, tuple) else (b,)
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert torch.isfinite(x).all() and torch.isfinite(y).all()
        torch.testing.assert_close(x, y, rtol=rtol, atol=atol)


def _fd_vjp(f, prim, cot):
    out = []
    for i, p in enumerate(prim):
        g = torch.empty_like(p)
        for e in range(p.numel()):
            hi = [q.detach().clone() for q in prim]
            lo = [q.detach().clone() for q in prim]
            hi[i].reshape(-1)[e] += EPS
            lo[i].reshape(-1)[e] -= EPS
            g.reshape(-1)[e] = ((f(*hi) * cot).sum() - (f(*lo) * cot).sum()) / (2 * EPS)
        out.append(g)
    return tuple(out)


def _tangents(prim):
    return tuple(torch.linspace(-0.2 + 0.03 * k, 0.3 + 0.03 * k, p.numel(), device=p.device).reshape_as(p)
                 for k, p in enumerate(prim))


def _cotangent(out):
    return torch.linspace(-0.3, 0.4, out.numel(), device=out.device).reshape_as(out)


def check_jvp(name, observable, device):
    f, prim = function_and_primals(name, observable, device)
    tan = _tangents(prim)
    val, t = torch.func.jvp(f, prim, tan)
    _close(val, f(*prim))
    hi = tuple(p + EPS * d for p, d in zip(prim, tan))
    lo = tuple(p - EPS * d for p, d in zip(prim, tan))
    fd = (f(*hi) - f(*lo)) / (2 * EPS)
    assert fd.abs().max() > 1e-6 and t.abs().max() > 0.1 * fd.abs().max()
    _close(t, fd, rtol=5e-2, atol=1e-4)


def check_vjp(name, observable, device):
    f, prim = function_and_primals(name, observable, device)
    out, pull = torch.func.vjp(f, *prim)
    eager = tuple(p.detach().clone().requires_grad_() for p in prim)
    eo = f(*eager)
    _close(out, eo)
    cot = _cotangent(out)
    got = pull(cot)
    want = torch.autograd.grad(eo, eager, grad_outputs=cot)
    _close(got, want)
    _close(want, _fd_vjp(f, prim, cot), rtol=5e-2, atol=5e-3)


def check_jacrev(name, observable, device):
    f, prim = function_and_primals(name, observable, device)
    got = torch.func.jacrev(f, argnums=tuple(range(len(prim))))(*prim)
    eager = tuple(p.detach().clone().requires_grad_() for p in prim)
    want = torch.autograd.functional.jacobian(f, eager)
    _close(got, want)


def check_vmap(name, observable, device, batch: int = 2):
    params, _ = CASES[name]
    fn = target(name, observable)
    x = scores(name, device, batch=batch)
    g = torch.Generator(device="cpu").manual_seed(7100 + batch + OBSERVABLES.index(observable))
    xs = x.unsqueeze(0) + (0.05 * torch.randn(3, *x.shape, generator=g)).to(device)
    kw = dict(params)
    got = torch.vmap(lambda p: fn(p, **kw))(xs)
    want = torch.stack([fn(p, **kw) for p in xs])
    _close(got, want)


def check_eager_backward(name, observable, device):
    f, prim = function_and_primals(name, observable, device)
    eager = tuple(p.detach().clone().requires_grad_() for p in prim)
    out = f(*eager)
    cot = _cotangent(out)
    (out * cot).sum().backward()
    got = tuple(p.grad for p in eager)
    assert all(g is not None for g in got)
    _close(got, _fd_vjp(f, prim, cot), rtol=5e-2, atol=5e-3)


def check_parameter_vmap_guard(name, observable, device):
    params, raw = CASES[name]
    fn = target(name, observable)
    x = scores(name, device)
    for (pname, value), rname in zip(params, raw):
        kw = dict(params)
        kw.pop(pname)
        mapped = torch.tensor((value, value + 0.1), device=device)
        try:
            torch.vmap(lambda p: fn(x, **kw, **{pname: p}))(mapped)
        except RuntimeError as e:
            msg = str(e)
            assert f"orihime::{name}_forward_t" in msg and f"mapping scalar argument {rname!r}" in msg, msg
            assert "keep scalar parameters unbatched" in msg and ".item()" not in msg, msg
        else:
            raise AssertionError(f"{name} {observable}: a mapped {pname} must raise")


def check_forward_mode_under_vmap_raises(name, observable, device):
    params, _ = CASES[name]
    fn = target(name, observable)
    x = scores(name, device)
    kw = dict(params)
    f = lambda p: fn(p, **kw)  # noqa: E731
    for how in ("jacfwd", "vmap_jvp"):
        try:
            if how == "jacfwd":
                torch.func.jacfwd(f)(x)
            else:
                xs = torch.stack((x, x + 0.05))
                ts = torch.stack((torch.ones_like(x), torch.linspace(-0.2, 0.3, x.numel(), device=device).reshape_as(x)))
                torch.vmap(lambda a, b: torch.func.jvp(f, (a,), (b,))[1])(xs, ts)
        except NotImplementedError as e:
            assert "jvp function" in str(e), str(e)
        else:
            raise AssertionError(f"{name} {observable}: {how} must raise NotImplementedError")


def check_entropy_parameter_directions_raise(name, device):
    params, _ = CASES[name]
    fn = target(name, "entropy")
    x = scores(name, device)
    for pname, value in params:
        kw = dict(params)
        kw.pop(pname)
        f = lambda p, d: fn(p, **kw, **{pname: d})  # noqa: E731
        d = torch.tensor(value, device=device)
        for how in ("jvp", "backward"):
            try:
                if how == "jvp":
                    torch.func.jvp(f, (x, d), (torch.zeros_like(x), torch.ones_like(d)))
                else:
                    f(x, d.clone().requires_grad_()).sum().backward()
            except NotImplementedError as e:
                msg = str(e)
                assert f"{name}_entropy" in msg, msg
                assert f"parameter {pname}" in msg and "finite differences" in msg, msg
            else:
                raise AssertionError(f"{name} entropy: the {pname} direction ({how}) must raise")


def run_all(names, device):
    """Every check for every family in `names`; returns the number run."""
    n = 0
    for name in names:
        for obs in OBSERVABLES:
            for chk in (check_jvp, check_vjp, check_jacrev, check_vmap, check_eager_backward,
                        check_parameter_vmap_guard, check_forward_mode_under_vmap_raises):
                chk(name, obs, device)
                n += 1
            check_vmap(name, obs, device, batch=1)
            n += 1
        check_entropy_parameter_directions_raise(name, device)
        n += 1
    return n


def check_masked_and_ragged(name, device):
    """A -inf mask and `lengths` under vmap, jvp and vjp: the transformed
    calls equal the eager ones, and masked cells get zero derivatives."""
    params, _ = CASES[name]
    kw = dict(params)
    x = scores(name, device)
    mask = torch.zeros_like(x, dtype=torch.bool)
    mask[:, 2, 0] = True
    mask[0, 0, 2] = True
    ln = torch.tensor([[3, 3], [2, 3]], dtype=torch.int32, device=device)
    for obs in OBSERVABLES:
        fn = target(name, obs)
        f = lambda p: fn(p, mask=mask, lengths=ln, **kw)  # noqa: E731
        xs = torch.stack((x, x + 0.05))
        _close(torch.vmap(f)(xs), torch.stack([f(p) for p in xs]))
        t = torch.linspace(-0.2, 0.3, x.numel(), device=device).reshape_as(x)
        val, tan = torch.func.jvp(f, (x,), (t,))
        _close(val, f(x))
        hi, lo = f(x + EPS * t), f(x - EPS * t)
        _close(tan, (hi - lo) / (2 * EPS), rtol=5e-2, atol=1e-4)
        out, pull = torch.func.vjp(f, x)
        cot = _cotangent(out)
        (g,) = pull(cot)
        xe = x.detach().clone().requires_grad_()
        (ge,) = torch.autograd.grad(f(xe), (xe,), grad_outputs=cot)
        _close(g, ge)
        assert bool((g[mask] == 0).all()) and bool((ge[mask] == 0).all())
        # vmap over the lengths (the scores unmapped), an empty pair included
        lns = torch.tensor([[[3, 3], [2, 3]], [[3, 2], [0, 3]]], dtype=torch.int32, device=device)
        got = torch.vmap(lambda l: fn(x, lengths=l, **kw))(lns)
        _close(got, torch.stack([fn(x, lengths=l.contiguous(), **kw) for l in lns]))
