"""Python drop-in for ``pyscx.accel.pca(..., device="gpu")`` on B200.

Mirrors the argument names, defaults, validation messages and AnnData output
contract of the reference binding (pyscx/src/accel/pca.rs:573-660 for the
signature and checks, :1137-1219 for ``write_pca_to_adata``).  All arithmetic
runs in libscxpca.so; PyTorch is used only to hold device buffers when the
caller passes CUDA tensors.  There is no CPU path: ``device="cpu"`` raises.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib

_MATH = {
    "strict_fp32": _lib.MATH_STRICT_FP32,
    "mixed_bf16": _lib.MATH_MIXED_BF16,
    "mixed_f16": _lib.MATH_MIXED_F16,
}
_QR = {"householder": _lib.QR_HOUSEHOLDER, "cholesky": _lib.QR_CHOLESKY}
_SPMM = {"default": _lib.SPMM_DEFAULT, "deterministic": _lib.SPMM_DETERMINISTIC,
         "benchmark_once": _lib.SPMM_DEFAULT}

BACKEND = "scx-b200"


@dataclass
class PcaResult:
    """Host result, the fields of PcaResult (scx-accel/src/pca/cpu.rs:84-110)
    plus singular values and the scaling statistics."""

    embeddings: object                      # (n_obs, n_components) float32 (numpy or torch)
    components: np.ndarray                  # (n_components, n_vars) float32
    variance_explained: np.ndarray          # (n_components,) float64
    variance_ratio: np.ndarray              # (n_components,) float64
    singular_values: np.ndarray             # (n_components,) float64
    mean: np.ndarray | None                 # (n_vars,) float64
    std: np.ndarray | None                  # (n_vars,) float64 when scaled
    n_components: int = 0
    n_obs: int = 0
    n_vars: int = 0
    total_var: float = 0.0
    total_var_recomputed: bool = False
    shifted_cholesky: int = 0
    eig_sweeps: int = 0
    resident_csr: bool = True
    n_shards: int = 0
    k: int = 0
    extra: dict = field(default_factory=dict)


# ---------------------------------------------------------------------------
# buffer helpers
# ---------------------------------------------------------------------------

def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _value_dtype(values) -> int:
    if _is_torch(values):
        import torch
        m = {torch.float32: _lib.F32, torch.bfloat16: _lib.BF16, torch.float16: _lib.F16}
        if values.dtype not in m:
            raise ValueError(f"unsupported value dtype {values.dtype}")
        return m[values.dtype]
    dt = np.asarray(values).dtype
    if dt == np.float32:
        return _lib.F32
    if dt == np.float16:
        return _lib.F16
    raise ValueError(f"unsupported value dtype {dt}; use float32 or float16")


def _ptr(x) -> int:
    if x is None:
        return 0
    if _is_torch(x):
        return int(x.data_ptr())
    return int(x.ctypes.data)


def _prepare_csr(indptr, indices, values, shape):
    """Return (Csr struct, keepalive tuple, memory kind, device ordinal)."""
    n_obs, n_vars = int(shape[0]), int(shape[1])
    if _is_torch(values):
        import torch
        if not values.is_cuda and values.dtype == torch.bfloat16:
            # host BF16 values (numpy has no bfloat16): passed by pointer, so a
            # pinned tensor is copied to the device at full link speed
            values = values.contiguous()
            indptr = np.ascontiguousarray(indptr.numpy() if _is_torch(indptr) else indptr, dtype=np.int64)
            indices = np.ascontiguousarray(indices.numpy() if _is_torch(indices) else indices, dtype=np.int32)
            if indptr.shape[0] != n_obs + 1:
                raise ValueError(f"indptr must have n_obs + 1 = {n_obs + 1} entries, got {indptr.shape[0]}")
            nnz = int(values.numel())
            if indices.shape[0] != nnz:
                raise ValueError("indices and values lengths differ")
            csr = _lib.Csr(n_obs, n_vars, nnz, _ptr(indptr), _ptr(indices), _ptr(values), _lib.BF16,
                           _lib.MEM_HOST)
            return csr, (indptr, indices, values), _lib.MEM_HOST, None
        if not values.is_cuda:
            values = values.numpy()
            indptr = indptr.numpy() if _is_torch(indptr) else indptr
            indices = indices.numpy() if _is_torch(indices) else indices
        else:
            indptr = indptr.to(torch.int64).contiguous()
            indices = indices.to(torch.int32).contiguous()
            values = values.contiguous()
            csr = _lib.Csr(n_obs, n_vars, int(values.numel()), _ptr(indptr), _ptr(indices),
                           _ptr(values), _value_dtype(values), _lib.MEM_DEVICE)
            return csr, (indptr, indices, values), _lib.MEM_DEVICE, values.device.index or 0
    indptr = np.ascontiguousarray(indptr, dtype=np.int64)
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    values = np.ascontiguousarray(values)
    if values.dtype not in (np.float32, np.float16):
        values = values.astype(np.float32)
    if indptr.shape[0] != n_obs + 1:
        raise ValueError(f"indptr must have n_obs + 1 = {n_obs + 1} entries, got {indptr.shape[0]}")
    nnz = int(values.shape[0])
    if indices.shape[0] != nnz:
        raise ValueError("indices and values lengths differ")
    csr = _lib.Csr(n_obs, n_vars, nnz, _ptr(indptr), _ptr(indices), _ptr(values),
                   _value_dtype(values), _lib.MEM_HOST)
    return csr, (indptr, indices, values), _lib.MEM_HOST, None


def _prepare_omega(omega, n_vars: int, k: int):
    """Explicit test matrix (n_vars x k) -> column-major float32 (pointer, memory, keepalive)."""
    if omega is None:
        return 0, _lib.MEM_HOST, None
    if _is_torch(omega) and omega.is_cuda:
        import torch
        if tuple(omega.shape) != (n_vars, k):
            raise ValueError(f"omega must have shape ({n_vars}, {k}), got {tuple(omega.shape)}")
        om = omega.to(torch.float32).t().contiguous()  # (k, n_vars) C-order == col-major
        return _ptr(om), _lib.MEM_DEVICE, om
    om = np.asarray(omega)
    if om.shape != (n_vars, k):
        raise ValueError(f"omega must have shape ({n_vars}, {k}), got {om.shape}")
    om = np.ascontiguousarray(om.astype(np.float32).T)
    return _ptr(om), _lib.MEM_HOST, om


def _prepare_gene_vector(v, n_vars: int, name: str):
    """A per-gene float64 vector -> (pointer, memory, keepalive); None -> (0, host, None)."""
    if v is None:
        return 0, _lib.MEM_HOST, None
    if _is_torch(v) and v.is_cuda:
        import torch
        t = v.detach().to(torch.float64).contiguous()
        if t.numel() != n_vars:
            raise ValueError(f"{name} must have n_vars = {n_vars} entries")
        return _ptr(t), _lib.MEM_DEVICE, t
    a = np.ascontiguousarray(np.asarray(v.detach().cpu() if _is_torch(v) else v, dtype=np.float64))
    if a.shape != (n_vars,):
        raise ValueError(f"{name} must have n_vars = {n_vars} entries")
    return _ptr(a), _lib.MEM_HOST, a


def _params(n_components, n_oversamples, n_power_iterations, zero_center, scale, clip_max, seed,
            qr_method, math_mode, spmm_policy, device):
    if qr_method not in _QR:
        raise ValueError(f"Invalid qr_method={qr_method!r}; expected 'householder' or 'cholesky'")
    if spmm_policy not in _SPMM:
        raise ValueError(f"Invalid spmm_policy={spmm_policy!r}; expected 'default', "
                         "'deterministic', or 'benchmark_once'")
    if math_mode not in _MATH:
        raise ValueError(f"Invalid math_mode={math_mode!r}; expected one of {sorted(_MATH)}")
    p = _lib.Params()
    p.n_components = int(n_components)
    p.n_oversamples = int(n_oversamples)
    p.n_power_iterations = int(n_power_iterations)
    p.zero_center = 1 if zero_center else 0
    p.scale = 1 if scale else 0
    p.clip_max = float(clip_max) if clip_max else 0.0
    p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    p.omega = None
    p.omega_memory = _lib.MEM_HOST
    p.qr_method = _QR[qr_method]
    p.math_mode = _MATH[math_mode]
    p.spmm_policy = _SPMM[spmm_policy]
    p.device_ordinal = int(device)
    p.stream = None
    return p


def _alloc_outputs(n_obs, n_vars, nc, device_embeddings, device):
    if device_embeddings:
        import torch
        emb = torch.empty((n_obs, nc), dtype=torch.float32, device=f"cuda:{device}")
    else:
        emb = np.empty((n_obs, nc), dtype=np.float32)
    comps = np.empty((nc, n_vars), dtype=np.float32)
    ve = np.empty(nc, dtype=np.float64)
    vr = np.empty(nc, dtype=np.float64)
    sv = np.empty(nc, dtype=np.float64)
    mean = np.empty(n_vars, dtype=np.float64)
    std = np.empty(n_vars, dtype=np.float64)
    res = _lib.Result()
    res.embeddings = _ptr(emb)
    res.components = _ptr(comps)
    res.variance_explained = _ptr(ve)
    res.variance_ratio = _ptr(vr)
    res.singular_values = _ptr(sv)
    res.mean = _ptr(mean)
    res.std = _ptr(std)
    res.embeddings_memory = _lib.MEM_DEVICE if device_embeddings else _lib.MEM_HOST
    return res, (emb, comps, ve, vr, sv, mean, std)


def _finish(res, bufs, n_obs, n_vars, nc, zero_center, scale, k):
    emb, comps, ve, vr, sv, mean, std = bufs
    return PcaResult(
        embeddings=emb, components=comps, variance_explained=ve, variance_ratio=vr,
        singular_values=sv, mean=mean if zero_center or scale else None,
        std=std if scale else None, n_components=nc, n_obs=n_obs, n_vars=n_vars,
        total_var=float(res.total_var), total_var_recomputed=bool(res.total_var_recomputed),
        shifted_cholesky=int(res.shifted_cholesky), resident_csr=bool(res.resident_csr),
        n_shards=int(res.n_shards), k=k,
        eig_sweeps=int(res.eig_sweeps))


# ---------------------------------------------------------------------------
# Array-level entry points
# ---------------------------------------------------------------------------

def randomized_pca(indptr, indices, values, shape, n_components: int = 50,
                   n_oversamples: int = 10, n_power_iterations: int = 2,
                   zero_center: bool = True, scale: bool = False, clip_max: float | None = None,
                   seed: int = 0, omega=None, qr_method: str = "householder",
                   math_mode: str = "strict_fp32", spmm_policy: str = "default",
                   device: int = 0, device_embeddings: bool = False,
                   embeddings_out=None, device_budget: int | None = None) -> PcaResult:
    """One-shot randomized PCA of a CSR matrix (host numpy or CUDA torch arrays).

    Same contract as ``scx_gpu::gpu_randomized_pca`` (scx-gpu/src/gpu_pca.rs:706-763)
    with an optional explicit ``omega`` (n_vars x k) and per-gene scaling.
    ``embeddings_out`` may be a preallocated (n_obs, n_components) float32
    buffer: a numpy array (e.g. pinned host memory) or a CUDA torch tensor.
    ``device_budget`` (bytes) caps the device memory of a host matrix's plan:
    a matrix whose resident plan does not fit is streamed from host memory in
    row shards (``resident_csr`` False), like the reference's streaming
    operator.
    """
    lib = _lib.load()
    csr, keep, mem, dev = _prepare_csr(indptr, indices, values, shape)
    if dev is not None:
        device = dev
    n_obs, n_vars = int(shape[0]), int(shape[1])
    p = _params(n_components, n_oversamples, n_power_iterations, zero_center, scale, clip_max,
                seed, qr_method, math_mode, spmm_policy, device)
    p.device_budget = int(device_budget or 0)
    k = min(int(n_components) + int(n_oversamples), n_vars, n_obs)
    optr, omem, okeep = _prepare_omega(omega, n_vars, k)
    p.omega = optr or None
    p.omega_memory = omem
    nc = int(n_components)
    if embeddings_out is not None:
        device_embeddings = _is_torch(embeddings_out) and embeddings_out.is_cuda
        res, bufs = _alloc_outputs(0, n_vars, max(nc, 0), False, device)
        res.embeddings = _ptr(embeddings_out)
        res.embeddings_memory = _lib.MEM_DEVICE if device_embeddings else _lib.MEM_HOST
        bufs = (embeddings_out,) + tuple(bufs[1:])
    else:
        res, bufs = _alloc_outputs(n_obs, n_vars, max(nc, 0), device_embeddings, device)
    err = _lib.errbuf()
    st = lib.scxpca_randomized(C.byref(csr), C.byref(p), C.byref(res), err, len(err))
    _lib.check(st, err)
    del keep, okeep
    return _finish(res, bufs, n_obs, n_vars, nc, zero_center, scale, k)


def preprocess(indptr, indices, values, shape, target_sum: float | None = 1e4, log1p: bool = True,
               row_factors=None, inplace: bool = False):
    """normalize_total(target_sum) + log1p (+ an explicit per-row factor) of a
    device CSR (CUDA torch tensors, float32 values) on the device
    (scxpca_preprocess; gpu_apply_fused_ops in scx-gpu/src/gpu_preprocess.rs).
    Returns the new values tensor (``values`` itself when ``inplace``)."""
    import torch
    lib = _lib.load()
    csr, keep, mem, dev = _prepare_csr(indptr, indices, values, shape)
    if mem != _lib.MEM_DEVICE:
        raise ValueError("preprocess needs CUDA tensors")
    vals = keep[2]
    if vals.dtype != torch.float32:
        raise ValueError("preprocess needs float32 values")
    out = vals if inplace else torch.empty_like(vals)
    rf = None
    if row_factors is not None:
        rf = row_factors.to(device=vals.device, dtype=torch.float32).contiguous()
        if rf.numel() != int(shape[0]):
            raise ValueError(f"row_factors must have n_obs = {int(shape[0])} entries")
    err = _lib.errbuf()
    st = lib.scxpca_preprocess(dev, C.byref(csr), _ptr(out), float(target_sum or 0.0), 1 if log1p else 0,
                               _ptr(rf) or None, None, err, len(err))
    _lib.check(st, err)
    return out


def project_columns(indptr, indices, values, shape, cols):
    """Keep the columns ``cols`` (sorted, unique) of a device CSR on the device
    (scxpca_project_columns; ProjectedShardSource in
    scx-accel/src/projected_source.rs).  Returns (indptr, indices, values, shape)."""
    import torch
    lib = _lib.load()
    csr, keep, mem, dev = _prepare_csr(indptr, indices, values, shape)
    if mem != _lib.MEM_DEVICE:
        raise ValueError("project_columns needs CUDA tensors")
    c = np.ascontiguousarray(np.asarray(cols.cpu() if _is_torch(cols) else cols), dtype=np.int32)
    d = keep[2].device
    out_ip = torch.empty(int(shape[0]) + 1, dtype=torch.int64, device=d)
    nnz = C.c_int64()
    err = _lib.errbuf()
    st = lib.scxpca_project_columns(dev, C.byref(csr), _ptr(c), len(c), _ptr(out_ip), None, None, C.byref(nnz),
                                    None, err, len(err))
    _lib.check(st, err)
    out_ix = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=d)
    out_vv = torch.empty(max(nnz.value, 1), dtype=torch.float32, device=d)
    st = lib.scxpca_project_columns(dev, C.byref(csr), _ptr(c), len(c), _ptr(out_ip), _ptr(out_ix), _ptr(out_vv),
                                    C.byref(nnz), None, err, len(err))
    _lib.check(st, err)
    return out_ip, out_ix[: nnz.value], out_vv[: nnz.value], (int(shape[0]), len(c))


def pflog_prepare(indptr, indices, values, shape, alpha: float):
    """PFlog (v4) representation of a raw-count device CSR: (delta values,
    baseline) with delta = log1p(4 alpha x) and b_i = -(1 / n_vars) sum_j
    delta_ij (scxpca_pflog_prepare; pflog_baseline_from_raw in
    scx-accel/src/pflog.rs).  Returns CUDA tensors (float32 nnz, float64 n_obs)."""
    import torch
    lib = _lib.load()
    csr, keep, mem, dev = _prepare_csr(indptr, indices, values, shape)
    if mem != _lib.MEM_DEVICE:
        raise ValueError("pflog_prepare needs CUDA tensors")
    vals = keep[2]
    delta = torch.empty_like(vals)
    base = torch.empty(int(shape[0]), dtype=torch.float64, device=vals.device)
    err = _lib.errbuf()
    st = lib.scxpca_pflog_prepare(dev, C.byref(csr), 4.0 * float(alpha), _ptr(delta), _ptr(base), None, err,
                                  len(err))
    _lib.check(st, err)
    return delta, base


def pflog_pca(indptr, indices, values, shape, alpha: float, n_components: int = 50, n_oversamples: int = 10,
              n_power_iterations: int = 2, zero_center: bool = True, seed: int = 0, omega=None,
              qr_method: str = "householder", math_mode: str = "strict_fp32", device: int = 0,
              device_embeddings: bool = False):
    """Baseline-aware (PFlog v4) randomized PCA of raw counts on the GPU:
    delta = log1p(4 alpha x) and the per-cell baseline on the device, then the
    PCA of Z = delta + baseline 1^T without densifying it (scxpca_pflog_pca;
    pflog_pca in scx-accel/src/pca/cpu.rs, which the reference runs on the
    CPU).  ``values`` are raw counts (host numpy or CUDA torch, float32).
    Returns (PcaResult, baseline as a CUDA float64 tensor)."""
    import torch
    lib = _lib.load()
    if not (_is_torch(values) and values.is_cuda):
        d = torch.device("cuda", int(device))
        indptr = torch.as_tensor(np.ascontiguousarray(indptr, dtype=np.int64)).to(d)
        indices = torch.as_tensor(np.ascontiguousarray(indices, dtype=np.int32)).to(d)
        values = torch.as_tensor(np.ascontiguousarray(values, dtype=np.float32)).to(d)
    delta, base = pflog_prepare(indptr, indices, values, shape, alpha)
    csr, keep, mem, dev = _prepare_csr(indptr, indices, delta, shape)
    n_obs, n_vars = int(shape[0]), int(shape[1])
    p = _params(n_components, n_oversamples, n_power_iterations, zero_center, False, None, seed, qr_method,
                math_mode, "default", dev)
    k = min(int(n_components) + int(n_oversamples), n_vars, n_obs)
    optr, omem, okeep = _prepare_omega(omega, n_vars, k)
    p.omega = optr or None
    p.omega_memory = omem
    nc = int(n_components)
    res, bufs = _alloc_outputs(n_obs, n_vars, max(nc, 0), device_embeddings, dev)
    err = _lib.errbuf()
    st = lib.scxpca_pflog_pca(C.byref(csr), _ptr(base), _lib.MEM_DEVICE, C.byref(p), C.byref(res), err, len(err))
    _lib.check(st, err)
    del keep, okeep
    return _finish(res, bufs, n_obs, n_vars, nc, zero_center, False, k), base


def last_call_phases() -> dict:
    """Phases of this thread's last one-shot call (scxpca_last_call_phases):
    device ms per phase (upload, validate, stats, transform, pack, buffers,
    pca, download; destroy in host ms) and the call's host wall time."""
    lib = _lib.load()
    ms = np.zeros(len(_lib.PHASES), dtype=np.float64)
    wall = C.c_double()
    lib.scxpca_last_call_phases(_ptr(ms), len(ms), C.byref(wall))
    out = {name: float(v) for name, v in zip(_lib.PHASES, ms)}
    out["wall"] = float(wall.value)
    return out


class Plan:
    """Resident plan: the CSR uploaded/borrowed once, buffers allocated once.

    Mirrors the resident operator of scx-gpu (gpu_pca_resident.rs:87-347) and
    exposes the PcaOperator seam (pca_operator.rs:69-79) on CUDA tensors.
    """

    def __init__(self, indptr, indices, values, shape, n_components: int = 50,
                 n_oversamples: int = 10, n_power_iterations: int = 2, zero_center: bool = True,
                 scale: bool = False, clip_max: float | None = None, seed: int = 0,
                 qr_method: str = "householder", math_mode: str = "strict_fp32",
                 spmm_policy: str = "default", device: int = 0, stream: int | None = None,
                 center=None, gene_scale=None, device_budget: int | None = None):
        """``stream`` is a raw ``cudaStream_t`` handle (e.g. ``torch.cuda.Stream().cuda_stream``)
        every kernel of this plan is ordered on; None lets the plan own a stream.

        ``center`` / ``gene_scale`` (n_vars float64, numpy or CUDA torch) make the
        plan's matrix the affine map (X - 1 center^T) diag(gene_scale), with no
        column means re-subtracted (scxpca_plan_create_affine); ``zero_center``,
        ``scale`` and ``clip_max`` are then ignored."""
        self._lib = _lib.load()
        csr, keep, mem, dev = _prepare_csr(indptr, indices, values, shape)
        if dev is not None:
            device = dev
        self.device = int(device)
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_components = int(n_components)
        self.zero_center = zero_center
        self.scale = scale
        self._params = _params(n_components, n_oversamples, n_power_iterations, zero_center,
                               scale, clip_max, seed, qr_method, math_mode, spmm_policy, device)
        if stream:
            self._params.stream = int(stream)
        self._params.device_budget = int(device_budget or 0)
        # a borrowed device CSR must live as long as the plan, and so must a
        # host CSR that the plan streams from
        self._keep = keep
        self.nnz = int(csr.nnz)
        handle = C.c_void_p()
        err = _lib.errbuf()
        if center is not None or gene_scale is not None:
            self._params.scale = 0
            self._params.clip_max = 0.0
            cptr, cmem, ckeep = _prepare_gene_vector(center, self.shape[1], "center")
            sptr, smem, skeep = _prepare_gene_vector(gene_scale, self.shape[1], "gene_scale")
            if cptr and sptr and cmem != smem:
                raise ValueError("center and gene_scale must both be host or both be device arrays")
            vmem = cmem if cptr else smem
            self.zero_center = center is not None
            self.scale = gene_scale is not None
            st = self._lib.scxpca_plan_create_affine(C.byref(csr), C.byref(self._params), cptr or None,
                                                     sptr or None, vmem, C.byref(handle), err, len(err))
            del ckeep, skeep
        else:
            st = self._lib.scxpca_plan_create(C.byref(csr), C.byref(self._params), C.byref(handle),
                                              err, len(err))
        _lib.check(st, err)
        self._h = handle
        k = C.c_int64()
        ld = C.c_int64()
        nbytes = C.c_int64()
        self._lib.scxpca_plan_info(self._h, C.byref(k), C.byref(ld), C.byref(nbytes))
        self.k, self.ld, self.device_bytes = int(k.value), int(ld.value), int(nbytes.value)

    def set_profiling(self, enable: bool = True) -> None:
        """Enable per-stage CUDA-event timing (resets the counters)."""
        self._lib.scxpca_plan_set_profiling(self._h, 1 if enable else 0)

    def profile(self) -> dict:
        """Per-stage launches and device ms accumulated since set_profiling()."""
        pr = _lib.Profile()
        self._lib.scxpca_plan_get_profile(self._h, C.byref(pr))
        return {
            "stages": {name: {"launches": int(pr.launches[i]), "device_ms": float(pr.device_ms[i])}
                       for i, name in enumerate(_lib.STAGES)},
            "kernel_launches": int(pr.kernel_launches),
            "runs": int(pr.runs),
        }

    def close(self):
        if getattr(self, "_h", None):
            self._lib.scxpca_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def run(self, seed: int | None = None, omega=None, n_power_iterations: int | None = None,
            device_embeddings: bool = False, embeddings_out=None) -> PcaResult:
        """Run the power loop; ``embeddings_out`` may be a preallocated
        (n_obs, n_components) float32 buffer (numpy or CUDA torch)."""
        p = _lib.Params.from_buffer_copy(self._params)
        if seed is not None:
            p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        if n_power_iterations is not None:
            p.n_power_iterations = int(n_power_iterations)
        optr, omem, okeep = _prepare_omega(omega, self.shape[1], self.k)
        p.omega = optr or None
        p.omega_memory = omem
        n_obs, n_vars = self.shape
        nc = self.n_components
        if embeddings_out is not None:
            device_embeddings = _is_torch(embeddings_out) and embeddings_out.is_cuda
        res, bufs = _alloc_outputs(0 if embeddings_out is not None else n_obs, n_vars, nc,
                                   device_embeddings and embeddings_out is None, self.device)
        if embeddings_out is not None:
            res.embeddings = _ptr(embeddings_out)
            res.embeddings_memory = _lib.MEM_DEVICE if device_embeddings else _lib.MEM_HOST
            bufs = (embeddings_out,) + tuple(bufs[1:])
        err = _lib.errbuf()
        st = self._lib.scxpca_plan_run(self._h, C.byref(p), C.byref(res), err, len(err))
        _lib.check(st, err)
        del okeep
        return _finish(res, bufs, n_obs, n_vars, nc, self.zero_center, self.scale, self.k)

    # ---- operator seam (CUDA torch tensors) ----
    def matmat(self, v):
        import torch
        y = torch.empty((self.shape[0], self.k), dtype=torch.float32, device=v.device)
        v = v.to(torch.float32).contiguous()
        err = _lib.errbuf()
        st = self._lib.scxpca_plan_matmat(self._h, _ptr(v), v.shape[1], _ptr(y), self.k, err, len(err))
        _lib.check(st, err)
        return y

    def rmatmat(self, q):
        import torch
        z = torch.empty((self.shape[1], self.k), dtype=torch.float64, device=q.device)
        q = q.to(torch.float32).contiguous()
        err = _lib.errbuf()
        st = self._lib.scxpca_plan_rmatmat(self._h, _ptr(q), q.shape[1], _ptr(z), self.k, err, len(err))
        _lib.check(st, err)
        return z

    def qr(self, a):
        """Orthonormalise the columns of a CUDA float32 (m, k) tensor in place."""
        err = _lib.errbuf()
        st = self._lib.scxpca_plan_qr(self._h, _ptr(a), a.shape[0], a.stride(0), err, len(err))
        _lib.check(st, err)
        return a

    def backward(self, scores, grad_scores, solve_iterations: int = 8):
        """Gradients of a loss of the last run's scores (scxpca_plan_backward).

        ``scores`` and ``grad_scores`` are CUDA float32 (n_obs, n_components)
        tensors; returns (grad_values (nnz,) float32, grad_center (n_vars,)
        float64, grad_scale (n_vars,) float64), all CUDA tensors."""
        import torch
        dev = scores.device
        s = scores.to(torch.float32).contiguous()
        gs = grad_scores.to(device=dev, dtype=torch.float32).contiguous()
        if tuple(s.shape) != (self.shape[0], self.n_components) or s.shape != gs.shape:
            raise ValueError(f"scores and grad_scores must be ({self.shape[0]}, {self.n_components})")
        gv = torch.empty(max(self.nnz, 1), dtype=torch.float32, device=dev)
        gc = torch.empty(self.shape[1], dtype=torch.float64, device=dev)
        gsc = torch.empty(self.shape[1], dtype=torch.float64, device=dev)
        err = _lib.errbuf()
        st = self._lib.scxpca_plan_backward(self._h, _ptr(s), _ptr(gs), int(solve_iterations), _ptr(gv),
                                            _ptr(gc), _ptr(gsc), err, len(err))
        _lib.check(st, err)
        return gv[: self.nnz], gc, gsc

    def col_stats(self):
        n_vars = self.shape[1]
        s = np.empty(n_vars, dtype=np.float64)
        q = np.empty(n_vars, dtype=np.float64)
        err = _lib.errbuf()
        st = self._lib.scxpca_plan_col_stats(self._h, _ptr(s), _ptr(q), err, len(err))
        _lib.check(st, err)
        return s, q


class Batch:
    """Independent randomized PCAs of the row segments of one CSR matrix
    (scxpca_batch_*): one resident plan per segment, all runs recorded into a
    single CUDA graph over parallel branches.  ``branches=b > 0`` runs whole
    segments per branch on b branches, ``-b`` the lockstep schedule (all
    segments take each power-loop step together) over b streams, and 0
    autotunes both.  ``run(use_graph=False)`` runs one plain plan call per
    segment instead, the loop a caller of the one-PCA API would write."""

    def __init__(self, indptr, indices, values, shape, segment_offsets, n_components: int = 30,
                 n_oversamples: int = 10, n_power_iterations: int = 3, zero_center: bool = True,
                 seed: int = 0, qr_method: str = "householder", math_mode: str = "mixed_bf16",
                 device: int = 0, branches: int = 0):
        self._lib = _lib.load()
        csr, keep, mem, dev = _prepare_csr(indptr, indices, values, shape)
        if dev is not None:
            device = dev
        self.device = int(device)
        self.shape = (int(shape[0]), int(shape[1]))
        self.n_components = int(n_components)
        offs = np.ascontiguousarray(np.asarray(segment_offsets, dtype=np.int64))
        self.offsets = offs
        self.n_segments = len(offs) - 1
        self._keep = keep
        p = _params(n_components, n_oversamples, n_power_iterations, zero_center, False, None, seed,
                    qr_method, math_mode, "default", device)
        handle = C.c_void_p()
        err = _lib.errbuf()
        st = self._lib.scxpca_batch_create(C.byref(csr), _ptr(offs), self.n_segments, C.byref(p),
                                           int(branches), C.byref(handle), err, len(err))
        _lib.check(st, err)
        self._h = handle
        nb = C.c_int32()
        nodes = C.c_int64()
        tuned = np.zeros(12, dtype=np.float64)
        self._lib.scxpca_batch_info(self._h, C.byref(nb), C.byref(nodes), _ptr(tuned))
        # branches < 0: the lockstep schedule over -branches streams
        self.branches, self.graph_nodes = int(nb.value), int(nodes.value)
        self.lockstep = self.branches < 0
        cand = (1, 2, 4, 8, 16, 32)
        self.tuned_ms = {b: float(t) for b, t in zip(cand, tuned[:6]) if t > 0}
        self.tuned_ms.update({-b: float(t) for b, t in zip(cand, tuned[6:]) if t > 0})

    def run(self, use_graph: bool = True, embeddings_out=None, components: bool = True):
        """Returns (embeddings, components [seg, nc, n_vars] or None, singular values
        [seg, nc], variance ratios [seg, nc], device ms)."""
        n, g = self.shape
        nc, ns = self.n_components, self.n_segments
        emb = embeddings_out if embeddings_out is not None else np.empty((n, nc), dtype=np.float32)
        mem = _lib.MEM_DEVICE if (_is_torch(emb) and emb.is_cuda) else _lib.MEM_HOST
        comps = np.empty((ns, nc, g), dtype=np.float32) if components else None
        sv = np.empty((ns, nc), dtype=np.float64)
        vr = np.empty((ns, nc), dtype=np.float64)
        ms = C.c_double()
        err = _lib.errbuf()
        st = self._lib.scxpca_batch_run(self._h, 1 if use_graph else 0, _ptr(emb), mem, _ptr(comps),
                                        _ptr(sv), _ptr(vr), None, C.byref(ms), err, len(err))
        _lib.check(st, err)
        return emb, comps, sv, vr, float(ms.value)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.scxpca_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gaussian(n_rows: int, n_cols: int, seed: int, device: int = 0):
    """Seeded N(0,1) test matrix (n_rows x n_cols) as a CUDA float32 tensor."""
    import torch
    out = torch.empty((n_cols, n_rows), dtype=torch.float32, device=f"cuda:{device}")
    err = _lib.errbuf()
    st = _lib.load().scxpca_gaussian(device, int(seed) & 0xFFFFFFFFFFFFFFFF, n_rows, n_cols,
                                     _ptr(out), err, len(err))
    _lib.check(st, err)
    return out.t()


def wait_selftest(device: int = 0) -> None:
    """Run the give-up path of the bounded pipeline wait: a block whose
    mbarrier wait never completes.  Raises ScxPcaError with status TIMEOUT
    after about 1 s (the expected outcome); the device stays usable."""
    err = _lib.errbuf()
    st = _lib.load().scxpca_wait_selftest(device, err, len(err))
    _lib.check(st, err)


def synth_nb_csr_device(n_obs: int, n_vars: int, seed: int = 0, loc: float = -3.0,
                        dispersion: float = 0.3, device: int = 0):
    """Generate the synthetic NB CSR on the device; returns torch CUDA tensors."""
    import torch
    lib = _lib.load()
    dev = f"cuda:{device}"
    indptr = torch.empty(n_obs + 1, dtype=torch.int64, device=dev)
    nnz = C.c_int64()
    err = _lib.errbuf()
    st = lib.scxpca_synth_nb_csr(device, seed, n_obs, n_vars, loc, dispersion, _ptr(indptr), None,
                                 None, C.byref(nnz), err, len(err))
    _lib.check(st, err)
    indices = torch.empty(max(nnz.value, 1), dtype=torch.int32, device=dev)
    values = torch.empty(max(nnz.value, 1), dtype=torch.float32, device=dev)
    st = lib.scxpca_synth_nb_csr(device, seed, n_obs, n_vars, loc, dispersion, _ptr(indptr),
                                 _ptr(indices), _ptr(values), C.byref(nnz), err, len(err))
    _lib.check(st, err)
    return indptr, indices[: nnz.value], values[: nnz.value]


# ---------------------------------------------------------------------------
# AnnData-facing drop-in (pyscx.accel.pca)
# ---------------------------------------------------------------------------

def _resolve_device(device: str) -> int:
    if device in ("gpu", "auto", "cuda"):
        return 0
    for pre in ("gpu:", "cuda:"):
        if isinstance(device, str) and device.startswith(pre):
            return int(device[len(pre):])
    if device == "cpu":
        raise ValueError("device='cpu' is not served by scx_b200: this package is the GPU path only")
    raise ValueError(f"Invalid device={device!r}; expected 'auto', 'gpu', or 'gpu:N'")


def _resolve_mask(adata, mask_var, n_vars):
    var = getattr(adata, "var", None)
    if mask_var is None:
        if var is not None and hasattr(var, "columns") and "highly_variable" in var.columns:
            return np.asarray(var["highly_variable"], dtype=bool), "highly_variable", True
        return None, None, False
    if isinstance(mask_var, str):
        if var is None or mask_var not in getattr(var, "columns", ()):
            raise ValueError(f"mask_var={mask_var!r} is not a column of adata.var")
        return np.asarray(var[mask_var], dtype=bool), mask_var, mask_var == "highly_variable"
    m = np.asarray(mask_var, dtype=bool)
    if m.shape != (n_vars,):
        raise ValueError(f"mask_var must have length n_vars={n_vars}")
    return m, None, False


def pca(adata, n_comps: int = 50, zero_center: bool = True, random_state: int = 0,
        n_oversamples: int = 10, n_power_iterations: int = 2, device: str = "auto",
        method: str = "auto", qr_method: str = "householder", prefer_format: str = "csr",
        allow_tf32: bool = False, spmm_policy: str = "default", memory_budget=None,
        mask_var=None, *, scale: bool = False, max_value: float | None = None, omega=None,
        math_mode: str | None = None):
    """``pyscx.accel.pca`` drop-in (pyscx/src/accel/pca.rs:573-1127) for device="gpu".

    Writes ``obsm["X_pca"]``, ``varm["PCs"]`` and ``uns["pca"]`` like
    ``write_pca_to_adata`` (pca.rs:1137-1219).  ``method`` is validated but, as
    on the reference GPU path, every method runs randomized PCA.
    ``allow_tf32=True`` selects the BF16 tensor-core path (``math_mode`` can
    name it directly).  ``scale``/``max_value`` apply scanpy ``pp.scale``
    implicitly, without densifying.  If ``adata`` is itself a scipy CSR matrix
    the :class:`PcaResult` is returned instead of written.
    """
    if method not in ("auto", "randomized", "covariance"):
        raise ValueError(f"Invalid method={method!r}; expected 'auto', 'randomized', or 'covariance'")
    if qr_method not in _QR:
        raise ValueError(f"Invalid qr_method={qr_method!r}; expected 'householder' or 'cholesky'")
    if spmm_policy not in _SPMM:
        raise ValueError(f"Invalid spmm_policy={spmm_policy!r}; expected 'default', "
                         "'deterministic', or 'benchmark_once'")
    if prefer_format != "csr":
        raise ValueError(
            "pyscx.accel.pca only supports prefer_format='csr' "
            f"(got {prefer_format!r}). The covariance build and randomized SpMM paths are "
            "row-major; CSC offers no measurable speed-up and is not implemented.")
    dev = _resolve_device(device)
    if math_mode is None:
        math_mode = "mixed_bf16" if allow_tf32 else "strict_fp32"
    import scipy.sparse as sp

    x = adata if sp.issparse(adata) else getattr(adata, "X")
    if not sp.issparse(x):
        x = sp.csr_matrix(np.asarray(x))
    x = sp.csr_matrix(x) if not sp.isspmatrix_csr(x) and not isinstance(x, sp.csr_array) else x
    n_obs, n_vars_full = x.shape
    mask, mask_name, use_hv = _resolve_mask(adata if not sp.issparse(adata) else None, mask_var,
                                            n_vars_full)
    cols = None
    if mask is not None:
        cols = np.flatnonzero(mask)
        x = x[:, cols]
    x = x.tocsr()
    x.sort_indices()
    res = randomized_pca(x.indptr, x.indices, x.data, x.shape, n_components=n_comps,
                         n_oversamples=n_oversamples, n_power_iterations=n_power_iterations,
                         zero_center=zero_center, scale=scale, clip_max=max_value,
                         seed=random_state, omega=omega, qr_method=qr_method,
                         math_mode=math_mode, spmm_policy=spmm_policy, device=dev)
    if sp.issparse(adata):
        return res
    adata.obsm["X_pca"] = np.asarray(res.embeddings, dtype=np.float32)
    pcs = np.zeros((n_vars_full, res.n_components), dtype=np.float32)
    if cols is None:
        pcs[:] = res.components.T
    else:
        pcs[cols] = res.components.T
    adata.varm["PCs"] = pcs
    adata.uns["pca"] = {
        "variance": res.variance_explained,
        "variance_ratio": res.variance_ratio,
        "backend": BACKEND,
        "params": {"zero_center": zero_center, "use_highly_variable": use_hv,
                   "mask_var": mask_name, "n_comps": n_comps},
    }
    acc = adata.uns.get("scx_accel", {}) if hasattr(adata.uns, "get") else {}
    acc = dict(acc)
    acc["pca"] = {"route": "gpu", "backend": BACKEND, "math_mode": math_mode,
                  "spmm_policy": spmm_policy, "qr_method": qr_method,
                  "resident_csr": res.resident_csr}
    adata.uns["scx_accel"] = acc
    return None
