"""Our CUDA path against the reference's own CUDA path on the same GPU.

The reference CUDA extension is built by ``make -C oracle refcuda`` from
``src/sw*/kernels_gpu.cu``, ``src/nw*/kernels_gpu.cu``,
``src/sv_*/kernels_gpu.cu`` and the op bodies beside them.  It has to be loaded before orihime_b200, which then takes over
the namespaced ``sw*`` / ``nw*`` / ``sv*`` ops; the reference's legacy
``soft_sw*`` / ``soft_nw*`` / ``soft_sv*`` ops stay the reference's CUDA path.  That
order is fixed per process, so the comparison runs in a child process.

Bar: values within rel 1e-5 of the reference CUDA path.  Maps and
second-order outputs must be at least as close to the fp64 oracle as the
reference CUDA path's own results (or within the 1e-5 / 1e-4 floors).  Our
distance to the reference CUDA path is printed with each case.
"""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
pytestmark = pytest.mark.gpu


def _worker():
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch
    from oracle import oracle as O

    torch.ops.load_library(O.ref_cuda_path())
    import orihime_b200  # noqa: F401  (takes over the namespaced ops)
    ops = torch.ops.orihime
    out = []

    def emb(B, N, M, seed, d=64):
        g = torch.Generator().manual_seed(seed)
        e, f = torch.randn(B, N, d, generator=g), torch.randn(B, M, d, generator=g)
        return (3 * torch.bmm(e, f.transpose(1, 2)) / d ** 0.5).float()

    def dist(a, b):
        return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max())

    for (B, N, M, T, seed) in [(3, 64, 80, 0.5, 1), (2, 200, 150, 0.7, 2), (2, 256, 256, 0.5, 3)]:
        s = emb(B, N, M, seed)
        sd = s.cuda()
        ln = torch.tensor([[N, M]] + [[N - 7, M - 13]] * (B - 1), dtype=torch.int32)
        rv, rm = ops.soft_sw_affine_float(sd, -2.0, -0.5, T, ln.cuda())[:2]
        ov, om = ops.sw_affine_forward(sd, -2.0, -0.5, T, ln.cuda())
        t64 = O.affine(s.numpy(), ln.numpy(), -2.0, -0.5, T, dtype=np.float64)
        rel = float(((ov - rv).abs() / rv.abs()).max())
        v = torch.randn(B, N, M, generator=torch.Generator().manual_seed(seed + 9))
        rh = ops.soft_sw_affine_hvp(sd, v.cuda(), -2.0, -0.5, T, ln.cuda())
        oh = ops.sw_affine_marginals_hvp(sd, v.cuda(), -2.0, -0.5, T, ln.cuda())
        h64 = O.affine_hvp(s.numpy(), v.numpy(), ln.numpy(), -2.0, -0.5, T, dtype=np.float64)
        rp = ops.soft_sw_affine_param_jacobian(sd, 2, -2.0, -0.5, T, ln.cuda())
        op_ = ops.sw_affine_marginals_grad_temp(sd, -2.0, -0.5, T, ln.cuda())
        p64 = O.affine_param_grad(s.numpy(), ln.numpy(), -2.0, -0.5, T, 2, dtype=np.float64)
        out.append(dict(case=[B, N, M, T], value_rel=rel,
                        map_ours_ref=dist(om.cpu(), rm.cpu()), map_ours_64=dist(om.cpu(), t64["map"]),
                        map_ref_64=dist(rm.cpu(), t64["map"]),
                        hvp_ours_ref=dist(oh.cpu(), rh.cpu()), hvp_ours_64=dist(oh.cpu(), h64),
                        hvp_ref_64=dist(rh.cpu(), h64), hvp_scale=float(np.abs(h64).max()),
                        dpdt_ours_ref=dist(op_.cpu(), rp.cpu()), dpdt_ours_64=dist(op_.cpu(), p64),
                        dpdt_ref_64=dist(rp.cpu(), p64), dpdt_scale=float(np.abs(p64).max())))
        # global alignment (soft Needleman-Wunsch, linear gap), same inputs
        rv, rm = ops.soft_nw_float(sd, -1.0, T, ln.cuda())[:2]
        ov, om = ops.nw_forward(sd, -1.0, T, ln.cuda())
        t64 = O.nw(s.numpy(), ln.numpy(), -1.0, T, dtype=np.float64)
        rel = float(((ov - rv).abs() / rv.abs()).max())
        rh = ops.soft_nw_hvp(sd, v.cuda(), -1.0, T, ln.cuda())
        oh = ops.nw_marginals_hvp(sd, v.cuda(), -1.0, T, ln.cuda())
        h64 = O.nw_hvp(s.numpy(), v.numpy(), ln.numpy(), -1.0, T, dtype=np.float64)
        rp = ops.soft_nw_param_jacobian(sd, 1, -1.0, T, ln.cuda())
        op_ = ops.nw_marginals_grad_temp(sd, -1.0, T, ln.cuda())
        p64 = O.nw_param_grad(s.numpy(), ln.numpy(), -1.0, T, 1, dtype=np.float64)
        out.append(dict(case=["nw", B, N, M, T], value_rel=rel,
                        map_ours_ref=dist(om.cpu(), rm.cpu()), map_ours_64=dist(om.cpu(), t64["map"]),
                        map_ref_64=dist(rm.cpu(), t64["map"]),
                        hvp_ours_ref=dist(oh.cpu(), rh.cpu()), hvp_ours_64=dist(oh.cpu(), h64),
                        hvp_ref_64=dist(rh.cpu(), h64), hvp_scale=float(np.abs(h64).max()),
                        dpdt_ours_ref=dist(op_.cpu(), rp.cpu()), dpdt_ours_64=dist(op_.cpu(), p64),
                        dpdt_ref_64=dist(rp.cpu(), p64), dpdt_scale=float(np.abs(p64).max())))
        # global alignment with affine gaps, same inputs
        rv, rm = ops.soft_nw_affine_float(sd, -2.0, -0.5, T, ln.cuda())[:2]
        ov, om = ops.nw_affine_forward(sd, -2.0, -0.5, T, ln.cuda())
        t64 = O.nw_affine(s.numpy(), ln.numpy(), -2.0, -0.5, T, dtype=np.float64)
        rel = float(((ov - rv).abs() / rv.abs().clamp_min(1.0)).max())
        rh = ops.soft_nw_affine_hvp(sd, v.cuda(), -2.0, -0.5, T, ln.cuda())
        oh = ops.nw_affine_marginals_hvp(sd, v.cuda(), -2.0, -0.5, T, ln.cuda())
        h64 = O.nw_affine_hvp(s.numpy(), v.numpy(), ln.numpy(), -2.0, -0.5, T, dtype=np.float64)
        rp = ops.soft_nw_affine_param_jacobian(sd, 2, -2.0, -0.5, T, ln.cuda())
        op_ = ops.nw_affine_marginals_grad_temp(sd, -2.0, -0.5, T, ln.cuda())
        p64 = O.nw_affine_param_grad(s.numpy(), ln.numpy(), -2.0, -0.5, T, 2, dtype=np.float64)
        out.append(dict(case=["nw_affine", B, N, M, T], value_rel=rel,
                        map_ours_ref=dist(om.cpu(), rm.cpu()), map_ours_64=dist(om.cpu(), t64["map"]),
                        map_ref_64=dist(rm.cpu(), t64["map"]),
                        hvp_ours_ref=dist(oh.cpu(), rh.cpu()), hvp_ours_64=dist(oh.cpu(), h64),
                        hvp_ref_64=dist(rh.cpu(), h64), hvp_scale=float(np.abs(h64).max()),
                        dpdt_ours_ref=dist(op_.cpu(), rp.cpu()), dpdt_ours_64=dist(op_.cpu(), p64),
                        dpdt_ref_64=dist(rp.cpu(), p64), dpdt_scale=float(np.abs(p64).max())))
        # Saigo-Vert, affine and linear gaps, same inputs
        for lin in (False, True):
            if lin:
                rv, rm = ops.soft_sv_linear_float(sd, -1.0, T, ln.cuda())[:2]
                ov, om = ops.sv_linear_forward(sd, -1.0, T, ln.cuda())
                rh = ops.soft_sv_linear_hvp(sd, v.cuda(), -1.0, T, ln.cuda())
                oh = ops.sv_linear_marginals_hvp(sd, v.cuda(), -1.0, T, ln.cuda())
                rp = ops.soft_sv_linear_param_jacobian(sd, 1, -1.0, T, ln.cuda())
                op_ = ops.sv_linear_marginals_grad_temp(sd, -1.0, T, ln.cuda())
                g3 = (-1.0, -1.0, T)
            else:
                rv, rm = ops.soft_sv_affine_float(sd, -2.0, -0.5, T, ln.cuda())[:2]
                ov, om = ops.sv_affine_forward(sd, -2.0, -0.5, T, ln.cuda())
                rh = ops.soft_sv_affine_hvp(sd, v.cuda(), -2.0, -0.5, T, ln.cuda())
                oh = ops.sv_affine_marginals_hvp(sd, v.cuda(), -2.0, -0.5, T, ln.cuda())
                rp = ops.soft_sv_affine_param_jacobian(sd, 2, -2.0, -0.5, T, ln.cuda())
                op_ = ops.sv_affine_marginals_grad_temp(sd, -2.0, -0.5, T, ln.cuda())
                g3 = (-2.0, -0.5, T)
            t64 = O.sv(s.numpy(), ln.numpy(), *g3, linear=lin, dtype=np.float64)
            rel = float(((ov - rv).abs() / rv.abs().clamp_min(1.0)).max())
            h64 = O.sv_hvp(s.numpy(), v.numpy(), ln.numpy(), *g3, dtype=np.float64)
            p64 = O.sv_param_grad(s.numpy(), ln.numpy(), *g3, 1 if lin else 2, linear=lin,
                                  dtype=np.float64)
            out.append(dict(case=["sv_linear" if lin else "sv_affine", B, N, M, T], value_rel=rel,
                            map_ours_ref=dist(om.cpu(), rm.cpu()), map_ours_64=dist(om.cpu(), t64["map"]),
                            map_ref_64=dist(rm.cpu(), t64["map"]),
                            hvp_ours_ref=dist(oh.cpu(), rh.cpu()), hvp_ours_64=dist(oh.cpu(), h64),
                            hvp_ref_64=dist(rh.cpu(), h64), hvp_scale=float(np.abs(h64).max()),
                            dpdt_ours_ref=dist(op_.cpu(), rp.cpu()), dpdt_ours_64=dist(op_.cpu(), p64),
                            dpdt_ref_64=dist(rp.cpu(), p64), dpdt_scale=float(np.abs(p64).max())))
    # timing: C2 (64 x 1024^2) on both CUDA paths
    s = emb(64, 1024, 1024, 1).cuda()

    def t(fn, n=3):
        fn(); torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record(); torch.cuda.synchronize()
        return a.elapsed_time(b) / n
    cells = 64 * 1024 * 1024
    tr = t(lambda: ops.soft_sw_affine_float(s, -2.0, -0.5, 0.5, None), 2)
    to = t(lambda: ops.sw_affine_forward(s, -2.0, -0.5, 0.5, None), 5)
    out.append(dict(timing="C2 64x1024^2 value+map", ref_ms=tr, ours_ms=to,
                    ref_gcups=cells / tr / 1e6, ours_gcups=cells / to / 1e6))
    tr = t(lambda: ops.soft_nw_float(s, -1.0, 0.5, None), 2)
    to = t(lambda: ops.nw_forward(s, -1.0, 0.5, None), 5)
    out.append(dict(timing="NW (global) 64x1024^2 value+map", ref_ms=tr, ours_ms=to,
                    ref_gcups=cells / tr / 1e6, ours_gcups=cells / to / 1e6))
    tr = t(lambda: ops.soft_nw_affine_float(s, -2.0, -0.5, 0.5, None), 2)
    to = t(lambda: ops.nw_affine_forward(s, -2.0, -0.5, 0.5, None), 5)
    out.append(dict(timing="NW affine 64x1024^2 value+map", ref_ms=tr, ours_ms=to,
                    ref_gcups=cells / tr / 1e6, ours_gcups=cells / to / 1e6))
    tr = t(lambda: ops.soft_sv_affine_float(s, -2.0, -0.5, 0.5, None), 2)
    to = t(lambda: ops.sv_affine_forward(s, -2.0, -0.5, 0.5, None), 5)
    out.append(dict(timing="Saigo-Vert affine 64x1024^2 value+map", ref_ms=tr, ours_ms=to,
                    ref_gcups=cells / tr / 1e6, ours_gcups=cells / to / 1e6))
    del s
    # C1: linear, 8 x 128^2, N(0,1) scores, gap -1, T 1
    s1 = torch.randn(8, 128, 128, generator=torch.Generator().manual_seed(0)).cuda()
    tr = t(lambda: ops.soft_sw_float(s1, -1.0, 1.0, None), 5)
    to = t(lambda: ops.sw_forward(s1, -1.0, 1.0, None), 5)
    cells = 8 * 128 * 128
    out.append(dict(timing="C1 linear 8x128^2 value+map", ref_ms=tr, ours_ms=to,
                    ref_gcups=cells / tr / 1e6, ours_gcups=cells / to / 1e6))
    # second-order ops at C5 shapes (256 x 512^2)
    s5 = torch.randn(256, 512, 512, generator=torch.Generator().manual_seed(5)).cuda()
    v5 = torch.randn_like(s5)
    cells = 256 * 512 * 512
    for name, rf, of in (
            ("C5 HVP", lambda: ops.soft_sw_affine_hvp(s5, v5, -2.0, -0.5, 0.5, None),
             lambda: ops.sw_affine_marginals_hvp(s5, v5, -2.0, -0.5, 0.5, None)),
            ("C5 dP/dT", lambda: ops.soft_sw_affine_param_jacobian(s5, 2, -2.0, -0.5, 0.5, None),
             lambda: ops.sw_affine_marginals_grad_temp(s5, -2.0, -0.5, 0.5, None)),
            ("C5 marginals_backward", lambda: ops.soft_sw_affine_backward_full(s5, v5, -2.0, -0.5, 0.5, None),
             lambda: ops.sw_affine_marginals_backward(s5, v5, -2.0, -0.5, 0.5, None))):
        tr, to = t(rf, 1), t(of, 3)
        out.append(dict(timing=name + " 256x512^2", ref_ms=tr, ours_ms=to,
                        ref_gcups=cells / tr / 1e6, ours_gcups=cells / to / 1e6))
    for name, rf, of in (
            ("NW HVP", lambda: ops.soft_nw_hvp(s5, v5, -1.0, 0.5, None),
             lambda: ops.nw_marginals_hvp(s5, v5, -1.0, 0.5, None)),
            ("NW dP/dT", lambda: ops.soft_nw_param_jacobian(s5, 1, -1.0, 0.5, None),
             lambda: ops.nw_marginals_grad_temp(s5, -1.0, 0.5, None)),
            ("NW marginals_backward", lambda: ops.soft_nw_backward_full(s5, v5, -1.0, 0.5, None),
             lambda: ops.nw_marginals_backward(s5, v5, -1.0, 0.5, None)),
            ("NW affine HVP", lambda: ops.soft_nw_affine_hvp(s5, v5, -2.0, -0.5, 0.5, None),
             lambda: ops.nw_affine_marginals_hvp(s5, v5, -2.0, -0.5, 0.5, None)),
            ("NW affine dP/dT", lambda: ops.soft_nw_affine_param_jacobian(s5, 2, -2.0, -0.5, 0.5, None),
             lambda: ops.nw_affine_marginals_grad_temp(s5, -2.0, -0.5, 0.5, None)),
            ("NW affine marginals_backward",
             lambda: ops.soft_nw_affine_backward_full(s5, v5, -2.0, -0.5, 0.5, None),
             lambda: ops.nw_affine_marginals_backward(s5, v5, -2.0, -0.5, 0.5, None)),
            ("SV affine HVP", lambda: ops.soft_sv_affine_hvp(s5, v5, -2.0, -0.5, 0.5, None),
             lambda: ops.sv_affine_marginals_hvp(s5, v5, -2.0, -0.5, 0.5, None)),
            ("SV affine dP/dT", lambda: ops.soft_sv_affine_param_jacobian(s5, 2, -2.0, -0.5, 0.5, None),
             lambda: ops.sv_affine_marginals_grad_temp(s5, -2.0, -0.5, 0.5, None)),
            ("SV affine marginals_backward",
             lambda: ops.soft_sv_affine_backward_full(s5, v5, -2.0, -0.5, 0.5, None),
             lambda: ops.sv_affine_marginals_backward(s5, v5, -2.0, -0.5, 0.5, None))):
        tr, to = t(rf, 1), t(of, 3)
        out.append(dict(timing=name + " 256x512^2", ref_ms=tr, ours_ms=to,
                        ref_gcups=cells / tr / 1e6, ours_gcups=cells / to / 1e6))
    del s5, v5
    # C3: 4096 pairs, lengths log-uniform [32, 2048] (seed 3).  The reference
    # runs padded chunks of 64 pairs of similar size (with lengths); ours runs
    # the packed ragged batch in one plan.
    from orihime_b200 import ragged
    rng = np.random.default_rng(3)
    ln = np.rint(np.exp(rng.uniform(np.log(32), np.log(2048), size=(4096, 2)))).astype(np.int64)
    order = np.argsort(-(ln[:, 0] * ln[:, 1]), kind="stable")
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    chunks = []
    for c0 in range(0, 4096, 64):
        idx = order[c0:c0 + 64]
        L1m, L2m = int(ln[idx, 0].max()), int(ln[idx, 1].max())
        sc = 3.0 * torch.randn(len(idx), L1m, L2m, generator=g, device="cuda")
        chunks.append((sc, torch.tensor(ln[idx], dtype=torch.int32, device="cuda")))
    cells = int((ln[:, 0] * ln[:, 1]).sum())

    def ref_c3():
        for sc, l in chunks:
            ops.soft_sw_affine_float(sc, -2.0, -0.5, 0.5, l)
    tr = t(ref_c3, 1)
    del chunks
    off, l32 = ragged.layout(ln)
    flat = 3.0 * torch.randn(int(off[-1]), generator=g, device="cuda")
    plan = ragged.Plan(l32, off, family="affine", device="cuda")
    to = t(lambda: plan.run(flat, gap_open=-2.0, gap_ext=-0.5, temp=0.5), 5)
    out.append(dict(timing="C3 4096 ragged pairs value+map+grads (reference: padded chunks of 64)",
                    ref_ms=tr, ours_ms=to, ref_gcups=cells / tr / 1e6, ours_gcups=cells / to / 1e6))
    print("RESULT " + json.dumps(out))


def test_against_reference_cuda_path():
    import torch
    from oracle import oracle as O

    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    if O.ref_cuda_path() is None:
        pytest.skip("reference CUDA extension not built (make -C oracle refcuda)")
    r = subprocess.run([sys.executable, __file__, "worker"], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    res = json.loads(r.stdout.split("RESULT ", 1)[1])
    for c in res:
        print(" ", c)
        if "timing" in c:
            continue
        assert c["value_rel"] <= 1e-5
        assert c["map_ours_64"] <= max(1e-5, c["map_ref_64"])
        assert c["hvp_ours_64"] <= max(1e-4 * c["hvp_scale"], c["hvp_ref_64"])
        assert c["dpdt_ours_64"] <= max(1e-4 * c["dpdt_scale"], c["dpdt_ref_64"])


if __name__ == "__main__" and len(sys.argv) > 1 and sys.argv[1] == "worker":
    _worker()
