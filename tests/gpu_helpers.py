"""Helpers for the GPU parity tests: run the engine (through the C ABI via neonufft_b200) and,
when it has been built, the reference's own GPU plans (oracle/_ref) on the same inputs."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent


def tdtypes(torch, dtype):
    if np.dtype(dtype) == np.float32:
        return torch.float32, torch.complex64, np.complex64
    return torch.float64, torch.complex128, np.complex128


def col_strides(modes):
    s = [1]
    for m in modes[:-1]:
        s.append(s[-1] * int(m))
    return s


def engine_t12(nnb, torch, dtype, sign, pts, inp, modes, tol, upsampfac, type_, order=1,
               opt_extra=None):
    rdt, cdt, npc = tdtypes(torch, dtype)
    loc = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.dtype(dtype))).cuda() for p in pts]
    opt = nnb.Options(tol=tol, upsampfac=upsampfac, order=order, **(opt_extra or {}))
    M = len(pts[0])
    plan = nnb.Plan(opt, sign, M, loc, modes)
    x = torch.from_numpy(np.ascontiguousarray(inp, dtype=npc)).cuda()
    strides = col_strides(modes)
    if type_ == 1:
        out = torch.zeros(int(np.prod(modes)), dtype=cdt, device="cuda")
        plan.transform_type_1(x, out, strides)
    else:
        out = torch.zeros(M, dtype=cdt, device="cuda")
        plan.transform_type_2(x, strides, out)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    plan.close()
    return res


def engine_t3(nnb, torch, dtype, sign, xin, xout, inp, tol, upsampfac=2.0, batch=1):
    rdt, cdt, npc = tdtypes(torch, dtype)
    a = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.dtype(dtype))).cuda() for p in xin]
    b = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.dtype(dtype))).cuda() for p in xout]
    opt = nnb.Options(tol=tol, upsampfac=upsampfac)
    M, K = len(xin[0]), len(xout[0])
    plan = nnb.PlanT3(opt, sign, M, a, K, b, batch_size=batch)
    x = torch.from_numpy(np.ascontiguousarray(inp, dtype=npc)).cuda()
    out = torch.zeros(K * batch, dtype=cdt, device="cuda")
    plan.add_input(x, M)
    plan.transform(out, K)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    plan.close()
    return res


class RefGpu:
    """The reference's own GPU plans compiled from its sources (oracle/_ref/libneonufft_ref.so)."""

    def __init__(self):
        from oracle import oracle as O
        self.ref = O.Ref()

    def t12(self, torch, dtype, sign, pts, inp, modes, tol, upsampfac, type_, order=1):
        rdt, cdt, npc = tdtypes(torch, dtype)
        loc = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.dtype(dtype))).cuda() for p in pts]
        x = torch.from_numpy(np.ascontiguousarray(inp, dtype=npc)).cuda()
        M = len(pts[0])
        n_out = int(np.prod(modes)) if type_ == 1 else M
        out = torch.zeros(n_out, dtype=cdt, device="cuda")
        torch.cuda.synchronize()
        lp = (C.c_void_p * 3)(*[t.data_ptr() for t in loc])
        md = (C.c_int64 * 3)(*[int(m) for m in modes])
        st = (C.c_int64 * 3)(*col_strides(modes))
        rc = self.ref.L.ref_gpu_type12(int(np.dtype(dtype) == np.float32), len(modes), type_, tol,
                                       upsampfac, sign, order, M, lp, md, x.data_ptr(),
                                       out.data_ptr(), st)
        assert rc == 0, f"reference GPU plan failed with code {rc}"
        torch.cuda.synchronize()
        return out.cpu().numpy()

    def t3(self, torch, dtype, sign, xin, xout, inp, tol, upsampfac=2.0, batch=1):
        rdt, cdt, npc = tdtypes(torch, dtype)
        a = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.dtype(dtype))).cuda() for p in xin]
        b = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.dtype(dtype))).cuda() for p in xout]
        x = torch.from_numpy(np.ascontiguousarray(inp, dtype=npc)).cuda()
        M, K = len(xin[0]), len(xout[0])
        out = torch.zeros(K * batch, dtype=cdt, device="cuda")
        torch.cuda.synchronize()
        pa = (C.c_void_p * 3)(*[t.data_ptr() for t in a])
        pb = (C.c_void_p * 3)(*[t.data_ptr() for t in b])
        rc = self.ref.L.ref_gpu_type3(int(np.dtype(dtype) == np.float32), len(xin), tol, upsampfac,
                                      sign, M, pa, K, pb, batch, x.data_ptr(), out.data_ptr())
        assert rc == 0, f"reference GPU type-3 plan failed with code {rc}"
        torch.cuda.synchronize()
        return out.cpu().numpy()


def ref_gpu_or_none():
    p = ROOT / "oracle" / "_ref" / "libneonufft_ref.so"
    if not p.exists():
        return None
    try:
        return RefGpu()
    except OSError:
        return None
