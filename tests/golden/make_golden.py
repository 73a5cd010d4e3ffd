"""Generate the golden fixtures in this folder from the reference itself.

Run on a machine that holds the reference sources: their root is the
environment variable ORIHIME_REFERENCE (default /root/reference).  It
copies the reference's Python package to a scratch
directory under /tmp, compiles the reference's CPU extension there with g++
(the source list of meson.build's ``cpp_sources``), imports it, and records
the public soft Smith-Waterman API's outputs on small seeded inputs:

* ``ohm.sw`` / ``sw_value`` / ``sw_entropy``, the ``sw_affine`` trio, the
  global-alignment ``nw`` and ``nw_affine`` trios and the Saigo-Vert ``sv``
  and ``sv_affine`` trios: forward results and the gradients of value, map
  (against a fixed cotangent) and entropy with respect to the pair scores;
* lengths-ragged and boolean-mask batches;
* tensor-valued (learnable) gap parameters and their gradients;
* ``ohm.ops.{sw,nw,sv}*.backward`` (map VJP) and
  ``.sensitivity`` (parameter fields).

Output: ``sw_golden.npz`` (float32 arrays, a few hundred KB).

    python tests/golden/make_golden.py
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
import sysconfig

import numpy as np

REF = os.environ.get("ORIHIME_REFERENCE", "/root/reference")
WORK = "/tmp/orihime_refpkg"
HERE = os.path.dirname(os.path.abspath(__file__))

CPP_SOURCES = [
    f"src/{m}/{f}"
    for m in ("cky", "sw", "sw_affine", "sv_affine", "sv_linear", "nw", "nw_affine", "dtw",
              "lev", "lcs", "osa", "damerau", "mas", "eisner")
    for f in ("registry.cpp", "torch_cpu.cpp", "kernels_cpu.cpp")
    if os.path.exists(os.path.join(REF, "src", m, f))
]


def build_reference() -> str:
    import torch

    pkg = os.path.join(WORK, "orihime")
    so = os.path.join(pkg, "_C.so")
    if os.path.exists(so):
        return WORK
    shutil.rmtree(WORK, ignore_errors=True)
    shutil.copytree(os.path.join(REF, "orihime"), pkg)
    tdir = os.path.dirname(torch.__file__)
    abi = int(torch._C._GLIBCXX_USE_CXX11_ABI)
    flags = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", f"-D_GLIBCXX_USE_CXX11_ABI={abi}",
             "-DUSE_TORCH_LIBRARY", f"-I{REF}/src", f"-I{tdir}/include",
             f"-I{tdir}/include/torch/csrc/api/include",
             f"-I{sysconfig.get_paths()['include']}"]
    objs = []

    def compile_one(src: str) -> str:
        obj = os.path.join(WORK, src.replace("/", "_") + ".o")
        subprocess.run(["g++", *flags, "-c", os.path.join(REF, src), "-o", obj], check=True)
        return obj

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(compile_one, CPP_SOURCES))
    subprocess.run(["g++", "-shared", "-fopenmp", *objs, f"-L{tdir}/lib", "-ltorch", "-ltorch_cpu",
                    "-lc10", "-ltorch_python", f"-Wl,-rpath,{tdir}/lib", "-o", so], check=True)
    return WORK


def seeded(shape, seed, scale=1.0):
    import torch

    g = torch.Generator().manual_seed(seed)
    return torch.randn(*shape, generator=g) * scale


def main() -> None:
    sys.path.insert(0, build_reference())
    import torch
    import orihime as ohm

    torch.set_num_threads(1)
    out: dict[str, np.ndarray] = {}

    def put(key, t):
        out[key] = t.detach().cpu().numpy().astype(np.float32) if hasattr(t, "detach") else np.asarray(t)

    cases = [
        # name, B, L1, L2, seed, lengths
        ("sq", 2, 9, 9, 11, None),
        ("rect", 3, 7, 12, 12, None),
        ("ragged", 4, 10, 13, 13, [[10, 13], [4, 9], [0, 5], [7, 1]]),
        ("unit", 2, 1, 1, 14, None),
        ("row", 2, 1, 11, 15, None),
    ]
    for name, B, L1, L2, seed, lens in cases:
        x0 = seeded((B, L1, L2), seed, 1.5)
        cot = seeded((B, L1, L2), seed + 100)
        lt = None if lens is None else torch.tensor(lens, dtype=torch.int32)
        put(f"{name}/scores", x0)
        put(f"{name}/cot", cot)
        if lt is not None:
            put(f"{name}/lengths", lt)
        for fam, kw in (("lin", dict(gap_score=-1.0, temperature=0.7)),
                        ("aff", dict(gap_open_score=-2.0, gap_extend_score=-0.5,
                                     temperature=0.7)),
                        ("nw", dict(gap_score=-1.0, temperature=0.7)),
                        ("nwa", dict(gap_open_score=-2.0, gap_extend_score=-0.5,
                                     temperature=0.7)),
                        ("svl", dict(gap_score=-1.0, temperature=0.7)),
                        ("sva", dict(gap_open_score=-2.0, gap_extend_score=-0.5,
                                     temperature=0.7))):
            fmap, fval, fent = {"lin": (ohm.sw, ohm.sw_value, ohm.sw_entropy),
                                "aff": (ohm.sw_affine, ohm.sw_affine_value, ohm.sw_affine_entropy),
                                "nw": (ohm.nw, ohm.nw_value, ohm.nw_entropy),
                                "nwa": (ohm.nw_affine, ohm.nw_affine_value,
                                        ohm.nw_affine_entropy),
                                "svl": (ohm.sv, ohm.sv_value, ohm.sv_entropy),
                                "sva": (ohm.sv_affine, ohm.sv_affine_value,
                                        ohm.sv_affine_entropy)}[fam]
            key = f"{name}/{fam}"
            x = x0.clone().requires_grad_(True)
            v = fval(x, lengths=lt, **kw)
            (g,) = torch.autograd.grad(-v.mean(), x)
            put(f"{key}/value", v)
            put(f"{key}/dvalue", g)
            x = x0.clone().requires_grad_(True)
            m = fmap(x, lengths=lt, **kw)
            (g,) = torch.autograd.grad((m * cot).sum(), x)
            put(f"{key}/map", m)
            put(f"{key}/dmap", g)
            x = x0.clone().requires_grad_(True)
            h = fent(x, lengths=lt, **kw)
            (g,) = torch.autograd.grad(h.sum(), x)
            put(f"{key}/entropy", h)
            put(f"{key}/dentropy", g)
            op = {"lin": ohm.ops.sw, "aff": ohm.ops.sw_affine, "nw": ohm.ops.nw,
                  "nwa": ohm.ops.nw_affine, "svl": ohm.ops.sv,
                  "sva": ohm.ops.sv_affine}[fam]
            sens = op.sensitivity(x0, lengths=lt, **kw)
            for k2, t in sens.items():
                put(f"{key}/sens_{k2}", t)
            bw = op.backward(x0, grad_map=cot, lengths=lt, **kw)
            for k2, t in bw.items():
                put(f"{key}/bw_{k2}", t)

    # boolean mask (True = excluded) and tensor-valued learnable parameters
    x0 = seeded((2, 8, 10), 21, 1.5)
    mask = torch.zeros(2, 8, 10, dtype=torch.bool)
    mask[0, :, 7:] = True
    mask[1, 5:, :] = True
    mask[1, 2, 3] = True
    put("mask/scores", x0)
    put("mask/mask", mask.to(torch.int32))
    for fam in ("lin", "aff", "nw"):
        x = x0.clone().requires_grad_(True)
        if fam in ("lin", "nw"):
            gp = torch.tensor(-1.0, requires_grad=True)
            tp = torch.tensor(0.8, requires_grad=True)
            fv = ohm.sw_value if fam == "lin" else ohm.nw_value
            v = fv(x, gap_score=gp, temperature=tp, mask=mask)
            grads = torch.autograd.grad(v.sum(), (x, gp, tp))
            names = ("dx", "dgap", "dtemp")
        else:
            go = torch.tensor(-2.0, requires_grad=True)
            ge = torch.tensor(-0.5, requires_grad=True)
            tp = torch.tensor(0.8, requires_grad=True)
            v = ohm.sw_affine_value(x, gap_open_score=go, gap_extend_score=ge, temperature=tp,
                                    mask=mask)
            grads = torch.autograd.grad(v.sum(), (x, go, ge, tp))
            names = ("dx", "dgap_open", "dgap_ext", "dtemp")
        put(f"mask/{fam}/value", v)
        for n_, g_ in zip(names, grads):
            put(f"mask/{fam}/{n_}", g_)
        m = {"lin": ohm.sw, "aff": ohm.sw_affine, "nw": ohm.nw}[fam](
            x0, mask=mask, **(dict(gap_score=-1.0, temperature=0.8) if fam != "aff" else
                             dict(gap_open_score=-2.0, gap_extend_score=-0.5, temperature=0.8)))
        put(f"mask/{fam}/map", m)

    dst = os.path.join(HERE, "sw_golden.npz")
    np.savez_compressed(dst, **out)
    print(f"wrote {dst}: {len(out)} arrays")


if __name__ == "__main__":
    main()
