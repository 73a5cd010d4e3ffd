"""torch.compile checks of the public functions (map, value, entropy),
shared by the CPU run (oracle-backed kernels, tests/_oracle_cpu_ops.py) and
the GPU run of tests/test_compile_observables.py.

They restate the reference's compile contract (tests/test_compile.py of
megure-labs/orihime): fullgraph and graph-break compiles under aot_eager and
the default inductor give the eager observables and primary gradients;
tensor parameters stay dynamic inputs of one compiled graph and get their
gradients (entropy: primary direction only); a -inf mask compiles too.
"""

from __future__ import annotations

import torch

import orihime_b200 as ohm
from _func_checks import CASES, target


def _close(a, b):
    torch.testing.assert_close(a, b, rtol=1e-4, atol=1e-5)


def _x(name, device, shape=(1, 4, 4)):
    g = torch.Generator(device="cpu").manual_seed(1234 + list(CASES).index(name))
    return torch.randn(*shape, generator=g).to(device)


def check_observables(name, device, backend, fullgraph):
    params, _ = CASES[name]
    kw = dict(params)
    x = _x(name, device)
    fns = [target(name, o) for o in ("map", "value", "entropy")]

    def obs(a):
        return tuple(f(a, **kw) for f in fns)

    torch._dynamo.reset()
    want = obs(x)
    comp = torch.compile(obs, backend=backend, fullgraph=fullgraph)
    for _ in range(2):   # repeatable
        for a, b in zip(comp(x), want):
            _close(a, b)


def check_reverse(name, observable, device, backend, fullgraph):
    params, _ = CASES[name]
    kw = dict(params)
    f = target(name, observable)

    def loss(a):
        return f(a, **kw).square().sum()

    torch._dynamo.reset()
    x = _x(name, device)
    a1, a2 = x.clone().requires_grad_(), x.clone().requires_grad_()
    l1 = loss(a1)
    l1.backward()
    l2 = torch.compile(loss, backend=backend, fullgraph=fullgraph)(a2)
    l2.backward()
    _close(l2, l1)
    _close(a2.grad, a1.grad)


def check_tensor_parameters(name, observable, device, backend="inductor"):
    params, _ = CASES[name]
    names = [n for n, _ in params]
    f = target(name, observable)

    def call(a, *ps):
        return f(a, **dict(zip(names, ps)))

    torch._dynamo.reset()
    x = _x(name, device)
    ps = [torch.tensor(v, device=device) for _, v in params]
    comp = torch.compile(call, backend=backend, fullgraph=True)
    _close(comp(x, *ps), call(x, *ps))
    for k in range(len(ps)):   # new parameter values reach the compiled graph
        changed = list(ps)
        changed[k] = changed[k] + 0.2
        want = call(x, *changed)
        assert not torch.allclose(want, call(x, *ps), rtol=1e-4, atol=1e-5)
        _close(comp(x, *changed), want)
    if observable == "entropy":
        return
    # reverse mode into the scores and every tensor parameter

    def loss(a, *qs):
        return call(a, *qs).square().sum()

    e = [x.clone().requires_grad_()] + [p.clone().requires_grad_() for p in ps]
    c = [x.clone().requires_grad_()] + [p.clone().requires_grad_() for p in ps]
    loss(*e).backward()
    torch._dynamo.reset()
    torch.compile(loss, backend=backend, fullgraph=True)(*c).backward()
    for a, b in zip(c, e):
        _close(a.grad, b.grad)


def check_masked(name, device, backend="aot_eager"):
    params, _ = CASES[name]
    kw = dict(params)
    x = _x(name, device, (2, 4, 5))
    mask = torch.zeros_like(x, dtype=torch.bool)
    mask[:, 3, 0] = True
    mask[1, 0, 4] = True
    ln = torch.tensor([[4, 5], [3, 4]], dtype=torch.int32, device=device)
    for obs in ("map", "value", "entropy"):
        f = target(name, obs)

        def loss(a):
            return f(a, mask=mask, lengths=ln, **kw).square().sum()

        torch._dynamo.reset()
        a1, a2 = x.clone().requires_grad_(), x.clone().requires_grad_()
        loss(a1).backward()
        l2 = torch.compile(loss, backend=backend, fullgraph=True)(a2)
        l2.backward()
        _close(a2.grad, a1.grad)
        assert bool((a2.grad[mask] == 0).all())


def run_all(names, device, backends=("aot_eager", "inductor")):
    n = 0
    for name in names:
        for backend in backends:
            for fg in (True, False):
                check_observables(name, device, backend, fg)
                n += 1
            for obs in ("map", "value", "entropy"):
                check_reverse(name, obs, device, backend, True)
                n += 1
        for obs in ("map", "value", "entropy"):
            check_tensor_parameters(name, obs, device, backends[-1])
            n += 1
        check_masked(name, device)
        n += 1
    return n
