"""Device CSR matrices: the BCOO operators of the reference, uploaded once.

The reference keeps every operator as a ``jax.experimental.sparse.BCOO`` built by
``_to_jax`` (amjax/multilevel.py:548-554).  Here an operator is an int32 CSR pattern
with FP64 and FP32 value copies in torch CUDA tensors; ``A @ x`` runs the library's SpMV.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import torch

from . import _native as N

_DT = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32}


def _canonical_csr(M) -> sp.csr_matrix:
    M = sp.csr_matrix(M)
    if not M.has_canonical_format:
        M = M.copy()
        M.sum_duplicates()
    M.sort_indices()
    return M


def validate_csr(indptr, indices, shape):
    """Host-side structural check (the device kernels trust their inputs)."""
    n_rows, n_cols = shape
    if len(indptr) != n_rows + 1:
        raise ValueError(f"rowptr has {len(indptr)} entries, expected {n_rows + 1}")
    if indptr[0] != 0 or np.any(np.diff(indptr) < 0):
        raise ValueError("rowptr must start at 0 and be non-decreasing")
    if indptr[-1] != len(indices):
        raise ValueError("rowptr[-1] does not match the number of column indices")
    if len(indices) and (indices.min() < 0 or indices.max() >= n_cols):
        raise ValueError("column index out of range")
    if len(indices) > np.iinfo(np.int32).max or n_rows > np.iinfo(np.int32).max:
        raise ValueError("matrix too large for int32 indices")


class CSRMatrix:
    """A device CSR operator with FP64 and/or FP32 values.

    ``dtype`` is the operator's nominal dtype (the reference hierarchy's dtype);
    ``val64`` / ``val32`` are both present for an FP64 hierarchy (the FP32 copy feeds the
    mixed-precision cycle) and only ``val32`` for an FP32 one.
    """

    def __init__(self, rowptr, col, val64, val32, shape, dtype, host=None):
        self.rowptr = rowptr
        self.col = col
        self.val64 = val64
        self.val32 = val32
        self.shape = tuple(int(s) for s in shape)
        self.dtype = dtype
        self._host = host
        self._desc = None

    # ------------------------------------------------------------ construction
    @classmethod
    def from_scipy(cls, M, dtype=None, device=None, keep_fp32=True):
        M = _canonical_csr(M)
        dtype = np.dtype(M.dtype if dtype is None else dtype)
        if dtype not in _DT:
            raise TypeError(f"unsupported dtype {dtype}")
        validate_csr(M.indptr, M.indices, M.shape)
        dev = torch.device("cuda") if device is None else torch.device(device)
        rowptr = torch.as_tensor(M.indptr.astype(np.int32)).to(dev)
        col = torch.as_tensor(M.indices.astype(np.int32)).to(dev)
        data = M.data.astype(dtype)
        v64 = torch.as_tensor(data.astype(np.float64)).to(dev) if dtype == np.float64 else None
        v32 = torch.as_tensor(data.astype(np.float32)).to(dev) if (keep_fp32 or dtype == np.float32) else None
        host = sp.csr_matrix((data, M.indices, M.indptr), shape=M.shape)
        return cls(rowptr, col, v64, v32, M.shape, dtype, host=host)

    @classmethod
    def from_any(cls, A, dtype=None, device=None):
        if isinstance(A, CSRMatrix):
            return A
        if sp.issparse(A):
            return cls.from_scipy(A, dtype=dtype, device=device)
        if isinstance(A, torch.Tensor):
            return cls.from_scipy(sp.csr_matrix(A.detach().cpu().numpy()), dtype=dtype, device=device)
        return cls.from_scipy(sp.csr_matrix(np.asarray(A)), dtype=dtype, device=device)

    def with_values(self, values: torch.Tensor) -> "CSRMatrix":
        """Same pattern, new values (1-D tensor in CSR order)."""
        values = values.detach()
        if values.numel() != self.nnz:
            raise ValueError(f"expected {self.nnz} values, got {values.numel()}")
        v64 = values.to(torch.float64).contiguous() if self.dtype == np.float64 else None
        v32 = values.to(torch.float32).contiguous()
        return CSRMatrix(self.rowptr, self.col, v64, v32, self.shape, self.dtype)

    # ------------------------------------------------------------ properties
    @property
    def nnz(self) -> int:
        return int(self.col.numel())

    nse = nnz

    @property
    def device(self):
        return self.rowptr.device

    def values(self, dtype=None):
        dt = self.dtype if dtype is None else np.dtype(dtype)
        return self.val64 if dt == np.float64 else self.val32

    def desc(self) -> N.amg_csr:
        if self._desc is None:
            d = N.amg_csr()
            d.n_rows, d.n_cols = self.shape
            d.nnz = self.nnz
            d.rowptr = self.rowptr.data_ptr()
            d.col = self.col.data_ptr() if self.nnz else 0
            d.val64 = self.val64.data_ptr() if self.val64 is not None else None
            d.val32 = self.val32.data_ptr() if self.val32 is not None else None
            self._desc = d
        return self._desc

    def to_scipy(self) -> sp.csr_matrix:
        if self._host is None:
            vals = self.values().detach().cpu().numpy()
            self._host = sp.csr_matrix((vals, self.col.cpu().numpy(), self.rowptr.cpu().numpy()), shape=self.shape)
        return self._host

    def todense(self):
        return torch.as_tensor(self.to_scipy().toarray(), device=self.device)

    def astype(self, dtype):
        return CSRMatrix.from_scipy(self.to_scipy(), dtype=dtype, device=self.device)

    @property
    def T(self):
        return CSRMatrix.from_scipy(self.to_scipy().T.tocsr(), dtype=self.dtype, device=self.device)

    def transpose(self):
        return self.T

    def __repr__(self):
        return f"CSRMatrix(shape={self.shape}, nnz={self.nnz}, dtype={self.dtype})"

    # ------------------------------------------------------------ products
    def matvec(self, x: torch.Tensor) -> torch.Tensor:
        """y = A x on the device (x: [n] or [n, k], FP64 or FP32)."""
        if not isinstance(x, torch.Tensor):
            x = torch.as_tensor(np.asarray(x), device=self.device)
        if x.device != self.device:
            x = x.to(self.device)
        if x.dtype not in (torch.float64, torch.float32):
            x = x.to(torch.float64)
        x = x.contiguous()
        k = 1 if x.dim() == 1 else int(x.shape[1])
        if x.shape[0] != self.shape[1]:
            raise ValueError(f"shape mismatch: {self.shape} @ {tuple(x.shape)}")
        if x.dtype == torch.float64 and self.val64 is None:
            x = x.to(torch.float32)
        y = torch.empty((self.shape[0],) + tuple(x.shape[1:]), dtype=x.dtype, device=self.device)
        dt = 0 if x.dtype == torch.float64 else 1
        N.call("amg_spmv", self.desc(), dt, N.ptr(x), N.ptr(y), k, N.stream_ptr())
        return y

    def __matmul__(self, x):
        return self.matvec(x)
