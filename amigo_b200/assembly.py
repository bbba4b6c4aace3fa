"""KKT assembly on the device: element Hessian blocks into the CSR values.

Mirrors the Hessian assembly of OptimizationProblem::hessian
(include/optimization_problem.h:1063-1088): the values zeroed, then every
component group's elements, in order, add their Hessian columns into the
fixed CSR pattern (ComponentGroup::add_hessian_kernel,
include/component_group.h:144-162, CSRMat::add_row,
include/csr_matrix.h:554-567). The library inverts that scatter once per
pattern and sums every CSR entry's contributions in the reference's order
with one thread per entry. The values are therefore bit-identical to the
reference's CPU assembly and need no atomics (the reference's GPU backend
uses atomicAdd). The result stays on the device and feeds
``SparseLDL.factor``.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _native

__all__ = ["CSRAssembly"]

_llp = ctypes.POINTER(ctypes.c_longlong)


class CSRAssembly:
    """Assembly plan for one CSR pattern and a list of component groups.

    ``groups``: one [nelem, ncomp] integer array of global variable indices
    per component group, in the order the reference adds the groups.
    """

    def __init__(self, rowp, cols, groups):
        self._lib = _native.load()
        self.rowp = np.ascontiguousarray(rowp, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)
        self.n = len(self.rowp) - 1
        self.nnz = int(self.rowp[-1])
        groups = [np.ascontiguousarray(np.asarray(g).reshape(len(g), -1), dtype=np.int32)
                  for g in groups]
        self.shapes = [g.shape for g in groups]
        nelems = np.array([g.shape[0] for g in groups] or [0], dtype=np.int32)
        ncomp = np.array([g.shape[1] for g in groups] or [0], dtype=np.int32)
        conn = np.ascontiguousarray(np.concatenate([g.ravel() for g in groups])
                                    if groups else np.zeros(1, np.int32), dtype=np.int32)
        h = ctypes.c_void_p()
        st = self._lib.b200ldl_assembly_create(
            ctypes.byref(h), self.n, self.rowp.ctypes.data_as(_native._i32p),
            self.cols.ctypes.data_as(_native._i32p), len(groups),
            nelems.ctypes.data_as(_native._i32p), ncomp.ctypes.data_as(_native._i32p),
            conn.ctypes.data_as(_native._i32p))
        if st != 0:
            msg = self._lib.b200ldl_assembly_last_error(h) if h else b""
            if h:
                self._lib.b200ldl_assembly_destroy(h)
            raise _native.NativeError(
                f"b200ldl_assembly_create failed with status {st}: {(msg or b'').decode()}", st)
        self._h = h
        info = (ctypes.c_longlong * 4)()
        self._lib.b200ldl_assembly_info(h, info, 4)
        self.kept, self.dropped, self.nvals = int(info[0]), int(info[1]), int(info[2])

    def close(self):
        if getattr(self, "_h", None):
            self._lib.b200ldl_assembly_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def plan(self):
        """(ptr [nnz + 1], src): CSR entry p sums blocks[src[ptr[p]:ptr[p+1]]]
        in that order, blocks being the groups' element blocks flattened one
        after another."""
        ptr = np.empty(self.nnz + 1, dtype=np.int64)
        src = np.empty(max(1, self.kept), dtype=np.int64)
        self._lib.b200ldl_assembly_plan(self._h, ptr.ctypes.data_as(_llp),
                                        src.ctypes.data_as(_llp))
        return ptr, src[: self.kept]

    def values(self, blocks, out=None):
        """The CSR values from the element blocks: a float64 CUDA tensor of
        all groups' [nelem, ncomp, ncomp] blocks flattened one after another
        (block[e, j, i] = column j, row i of element e's Hessian), or a list
        of per-group tensors. Returns (or fills) a CUDA tensor of nnz values,
        ordered on the tensor's current stream."""
        import torch

        if isinstance(blocks, (list, tuple)):
            blocks = torch.cat([b.reshape(-1) for b in blocks])
        if not (torch.is_tensor(blocks) and blocks.is_cuda and blocks.dtype == torch.float64):
            raise TypeError("blocks must be a float64 CUDA tensor")
        blocks = blocks.contiguous().reshape(-1)
        if blocks.numel() != self.nvals:
            raise ValueError(f"expected {self.nvals} block values, got {blocks.numel()}")
        if out is None:
            out = torch.empty(self.nnz, dtype=torch.float64, device=blocks.device)
        stream = torch.cuda.current_stream(blocks.device)
        st = self._lib.b200ldl_assembly_values(
            self._h, ctypes.c_void_p(blocks.data_ptr()), ctypes.c_void_p(out.data_ptr()),
            ctypes.c_void_p(stream.cuda_stream))
        if st != 0:
            msg = self._lib.b200ldl_assembly_last_error(self._h)
            raise _native.NativeError(f"assembly failed with status {st}: {msg.decode()}", st)
        return out
