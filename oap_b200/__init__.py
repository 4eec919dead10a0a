"""oap_b200: B200-native Arnoldi eigensolver hot path of oap.

The product is ``liboapb200.so`` (C ABI, ``include/oapb200.h``); this module
is a ctypes front end over it for Python callers, the tests and the
benchmark.  Device buffers are passed as raw pointers (e.g. from torch
tensors); nothing here computes on the host.  Importing works without a GPU;
every call needs the built library and raises if it is missing.
"""

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboapb200.so")
_LIB = None

(OK, ERR_ARG, ERR_CUDA, NOT_CONVERGED, ERR_TIMEOUT, ERR_BOUNDS, ERR_CALLBACK, ERR_NOMEM, ERR_BREAKDOWN,
 ERR_NONFINITE) = range(10)
F64, F32 = 0, 1
SORT = {"LM": 0, "LR": 1, "LI": 2, "SM": 3, "SR": 4, "SI": 5}
PREC_FP64, PREC_MIXED = 0, 1
PASS_BF16 = 2  # apply_block only: the BF16 hi planes of the operator copy
PASS_BF16_COARSE = 3  # apply_block only: the BF16 hi planes, X rounded to BF16 too
INIT_RANDOM, INIT_FIRST_VALUE_IS_ONE, INIT_USER = 0, 1, 2
ACT_LINEAR, ACT_SIGMOID, ACT_TANH, ACT_SIN = 0, 1, 2, 3  # oapb_activation
TYPE_EIGENVECTOR, TYPE_WV = 0, 1


class OapbError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        super().__init__("%s: %s (status %d)" % (where, status_string(status), status))


class Mat(C.Structure):
    """oapb_mat: host handle over device planes (reference layout)."""
    _fields_ = [("columns", C.c_uint32), ("rows", C.c_uint32),
                ("re", C.c_void_p), ("im", C.c_void_p), ("dtype", C.c_int32)]


class Config(C.Structure):
    _fields_ = [("n", C.c_uint32), ("hdim", C.c_uint32), ("wanted", C.c_uint32),
                ("is_complex", C.c_int32), ("sort", C.c_int32),
                ("precision", C.c_int32), ("init", C.c_int32),
                ("max_restarts", C.c_uint32), ("tolerance", C.c_double),
                ("rho", C.c_double), ("seed", C.c_uint64), ("profile", C.c_int32),
                ("fallback_random", C.c_int32), ("tensor_cores", C.c_int32),
                ("refine", C.c_int32), ("autotune", C.c_int32)]


class TraceRec(C.Structure):
    _fields_ = [("phase", C.c_int32), ("iteration", C.c_int32), ("passes", C.c_uint32),
                ("bf16_passes", C.c_uint32), ("residual", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("restarts", C.c_uint32), ("matvecs", C.c_uint32),
                ("block_matvecs", C.c_uint32), ("dgks_passes", C.c_uint32),
                ("refine_iterations", C.c_uint32), ("converged", C.c_int32),
                ("max_residual", C.c_double), ("seconds", C.c_double),
                ("matvec_seconds", C.c_double), ("matvec_timed", C.c_uint32),
                ("matvec_fp32", C.c_uint32), ("kernel_launches", C.c_uint64),
                ("block_seconds", C.c_double), ("block_timed", C.c_uint32),
                ("block_fp32_timed", C.c_uint32), ("block_fp32_seconds", C.c_double),
                ("block_fp32_width", C.c_uint32), ("fallbacks", C.c_uint32),
                ("matvec_variant", C.c_uint32), ("block_bf16", C.c_uint32),
                ("block_bf16_timed", C.c_uint32), ("block_bf16_seconds", C.c_double),
                ("eig_fast", C.c_uint32), ("block_i8", C.c_uint32), ("onchip", C.c_uint32),
                ("pass_kernel_seconds", C.c_double * 3), ("pass_kernel_timed", C.c_uint32 * 3),
                ("symtri", C.c_uint32)]


class BatchProblem(C.Structure):
    _fields_ = [("n", C.c_uint32), ("re", C.c_void_p), ("im", C.c_void_p),
                ("eigvec_re", C.c_void_p), ("eigvec_im", C.c_void_p)]


class BatchStats(C.Structure):
    _fields_ = [("problems", C.c_uint32), ("converged", C.c_uint32),
                ("matvecs", C.c_uint64), ("restarts", C.c_uint64),
                ("ctas", C.c_uint32), ("seconds", C.c_double),
                ("variant", C.c_uint32), ("threads", C.c_uint32), ("operator_bytes", C.c_uint64)]


MATVEC_FN = C.CFUNCTYPE(C.c_int, C.POINTER(Mat), C.POINTER(Mat), C.c_void_p,
                        C.c_int, C.c_void_p)


def lib():
    """Load liboapb200.so; raise (never fall back) when it is not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "liboapb200.so is not built (run python -m oap_b200.build); "
                "there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        vp = C.c_void_p
        L.oapb_status_string.restype = C.c_char_p
        L.oapb_status_string.argtypes = [C.c_int]
        for name, args in {
            "oapb_dot_product": [P(Mat), P(Mat), P(Mat), vp],
            "oapb_transpose": [P(Mat), P(Mat), vp],
            "oapb_conjugate_transpose": [P(Mat), P(Mat), vp],
            "oapb_magnitude": [P(C.c_double), P(Mat), vp],
            "oapb_sum": [P(C.c_double), P(C.c_double), P(Mat), vp],
            "oapb_tensor_product": [P(Mat), P(Mat), P(Mat), vp],
            "oapb_add": [P(Mat), P(Mat), P(Mat), vp],
            "oapb_substract": [P(Mat), P(Mat), P(Mat), vp],
            "oapb_multiply_re_constant": [P(Mat), P(Mat), C.c_double, vp],
            "oapb_multiply_constant": [P(Mat), P(Mat), C.c_double, C.c_double, vp],
            "oapb_set_vector": [P(Mat), C.c_uint32, P(Mat), C.c_uint32, vp],
            "oapb_get_vector": [P(Mat), C.c_uint32, P(Mat), C.c_uint32, vp],
            "oapb_set_identity": [P(Mat), vp],
            "oapb_set_diagonal": [P(Mat), C.c_double, C.c_double, vp],
            "oapb_set_zero_matrix": [P(Mat), vp],
            "oapb_qr_givens": [P(Mat), P(Mat), P(Mat), vp],
            "oapb_qr_householder": [P(Mat), P(Mat), P(Mat), vp],
            "oapb_qr_givens_noalloc": [P(Mat), P(Mat), P(Mat), vp],
            "oapb_selftest_bounded_wait": [C.c_uint32, C.c_int32, P(C.c_int32), vp],
            "oapb_arnoldi_set_gram_operator_host": [vp, vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64],
            "oapb_arnoldi_gram_stream_info": [vp, P(C.c_uint32), P(C.c_uint32), P(C.c_uint64)],
            "oapb_is_upper_triangular": [P(C.c_int), P(Mat), C.c_double, vp],
            "oapb_calc_triangular_h": [P(Mat), P(Mat), C.c_uint32, P(C.c_uint32), vp],
            "oapb_arnoldi_create": [P(vp), P(Config), vp],
            "oapb_arnoldi_destroy": [vp],
            "oapb_arnoldi_set_dense_operator": [vp, P(Mat)],
            "oapb_arnoldi_set_callback": [vp, MATVEC_FN, vp],
            "oapb_arnoldi_set_start_vector": [vp, vp, vp],
            "oapb_arnoldi_solve": [vp, P(C.c_double), P(C.c_double), P(C.c_double), P(Mat)],
            "oapb_arnoldi_solve_host": [vp, vp, vp, P(C.c_double), P(C.c_double),
                                        P(C.c_double), vp, vp],
            "oapb_arnoldi_get_stats": [vp, P(Stats)],
            "oapb_arnoldi_get_trace": [vp, P(TraceRec), C.c_uint32, P(C.c_uint32)],
            "oapb_arnoldi_set_profile": [vp, C.c_int32],
            "oapb_arnoldi_test_outcome": [vp, C.c_uint32, P(C.c_double)],
            "oapb_gram_build": [vp, C.c_uint32, C.c_uint32, vp, vp, vp],
            "oapb_gram_trim": [],
            "oapb_arnoldi_set_start_shifts": [vp, P(C.c_double), C.c_uint32],
            "oapb_arnoldi_apply_block": [vp, vp, vp, C.c_uint32, vp, vp, C.c_int32],
            "oapb_arnoldi_set_gram_operator": [vp, vp, C.c_uint32, C.c_uint32],
            "oapb_images_to_matrix": [vp, C.c_int32, C.c_uint32, C.c_uint32, vp, vp],
            "oapb_mlp_save": [vp, C.c_char_p],
            "oapb_mlp_load": [P(vp), C.c_char_p, C.c_uint64],
            "oapb_arnoldi_save": [vp, C.c_char_p],
            "oapb_arnoldi_load": [vp, C.c_char_p],
            "oapb_arnoldi_resume": [vp, P(C.c_double), P(C.c_double), P(C.c_double), P(Mat)],
            "oapb_mat_write": [C.c_char_p, P(Mat), vp],
            "oapb_mat_read_info": [C.c_char_p, P(C.c_uint32), P(C.c_uint32), P(C.c_int32), P(C.c_int32)],
            "oapb_mat_read": [C.c_char_p, P(Mat), vp],
            "oapb_param_operators": [vp, P(vp), C.c_uint32, vp, C.c_uint32, C.c_uint32, vp, vp],
            "oapb_mlp_create": [P(vp), P(C.c_uint32), C.c_uint32, C.c_uint64],
            "oapb_mlp_destroy": [vp],
            "oapb_mlp_forward": [vp, vp, C.c_uint32, vp, vp],
            "oapb_mlp_backward": [vp, vp, vp, C.c_uint32, P(C.c_double), vp],
            "oapb_mlp_adam_step": [vp, C.c_float, vp],
            "oapb_mlp_copy": [vp, C.c_int, vp, vp],
            "oapb_mlp_set_params": [vp, vp, vp],
            "oapb_mlp_set_activations": [vp, P(C.c_int32), C.c_uint32],
            "oapb_mlp_get_activations": [vp, P(C.c_int32), C.c_uint32],
            "oapb_arnoldi_solve_batched": [P(Config), P(BatchProblem), C.c_uint32,
                                           P(C.c_double), P(C.c_double), P(C.c_double),
                                           P(C.c_int32), P(BatchStats), vp],
        }.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.oapb_mlp_num_params.argtypes = [vp]
        L.oapb_mlp_num_params.restype = C.c_uint64
        L.oapb_mlp_num_layers.restype = C.c_uint32
        L.oapb_mlp_num_layers.argtypes = [vp, vp]
        L.oapb_arnoldi_config_default.argtypes = [P(Config)]
        L.oapb_arnoldi_config_default.restype = None
        _LIB = L
    return _LIB


def status_string(st):
    try:
        return lib().oapb_status_string(st).decode()
    except RuntimeError:
        return "status %d" % st


def check(st, where=""):
    if st != OK:
        raise OapbError(st, where)
    return st


# ---------------------------------------------------------------- torch glue
def mat(re, im=None, columns=None, rows=None):
    """Mat over torch tensors (FP64, contiguous, on the device).  A 2-D tensor
    of shape (rows, columns) maps to the reference's row-major layout; a 1-D
    tensor is a 1-column vector."""
    t = re if re is not None else im
    if t.dim() == 1:
        r, c = t.shape[0], 1
    else:
        r, c = t.shape
    for x in (re, im):
        if x is not None:
            assert x.is_contiguous() and x.is_cuda
    return Mat(columns or c, rows or r,
               re.data_ptr() if re is not None else None,
               im.data_ptr() if im is not None else None,
               F64 if t.dtype.is_floating_point and t.element_size() == 8 else F32)


def _stream(stream):
    if stream is None:
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return C.c_void_p(stream)


class Arnoldi:
    """CuHArnoldi over the C ABI (oapb_arnoldi_*)."""

    def __init__(self, n, hdim, wanted, is_complex=False, sort="LM",
                 precision=PREC_FP64, tolerance=1e-10, max_restarts=300,
                 rho=1.0 / 3.14, seed=1, init=INIT_RANDOM, stream=None,
                 profile=False, fallback_random=False, tensor_cores=True, refine=True, autotune=True):
        L = lib()
        cfg = Config()
        L.oapb_arnoldi_config_default(C.byref(cfg))
        cfg.n, cfg.hdim, cfg.wanted = n, hdim, wanted
        cfg.is_complex = int(bool(is_complex))
        cfg.sort = SORT[sort] if isinstance(sort, str) else int(sort)
        cfg.precision, cfg.init = precision, init
        cfg.max_restarts, cfg.tolerance, cfg.rho, cfg.seed = max_restarts, tolerance, rho, seed
        cfg.profile = int(bool(profile))
        cfg.fallback_random = int(bool(fallback_random))
        cfg.tensor_cores = int(bool(tensor_cores))
        cfg.refine = int(bool(refine))
        cfg.autotune = int(autotune) if not isinstance(autotune, bool) else int(autotune)
        self.cfg = cfg
        self.h = C.c_void_p()
        check(L.oapb_arnoldi_create(C.byref(self.h), C.byref(cfg), _stream(stream)),
              "oapb_arnoldi_create")
        self._cb = None

    def close(self):
        if self.h:
            lib().oapb_arnoldi_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_operator(self, are, aim=None):
        self._A = (are, aim)
        m = mat(are, aim)
        check(lib().oapb_arnoldi_set_dense_operator(self.h, C.byref(m)),
              "oapb_arnoldi_set_dense_operator")

    def set_callback(self, fn):
        """fn(w: Mat, v: Mat, type: int, stream: int) -> int"""
        def tramp(w, v, user, typ, stream):
            try:
                return int(fn(w.contents, v.contents, typ, stream) or 0)
            except Exception as e:  # reported by solve()
                self._cb_error = e
                return 1
        self._cb = MATVEC_FN(tramp)
        check(lib().oapb_arnoldi_set_callback(self.h, self._cb, None),
              "oapb_arnoldi_set_callback")

    def set_start_shifts(self, shifts):
        arr = (C.c_double * max(1, len(shifts)))(*[float(x) for x in shifts])
        check(lib().oapb_arnoldi_set_start_shifts(self.h, arr, len(shifts)),
              "oapb_arnoldi_set_start_shifts")

    def set_start_vector(self, re, im=None):
        check(lib().oapb_arnoldi_set_start_vector(
            self.h, C.c_void_p(re.data_ptr()),
            C.c_void_p(im.data_ptr()) if im is not None else None),
            "oapb_arnoldi_set_start_vector")

    def solve(self, vectors=None, allow_not_converged=False, _entry="oapb_arnoldi_solve"):
        k = self.cfg.wanted
        er, ei, rs = (C.c_double * k)(), (C.c_double * k)(), (C.c_double * k)()
        vm = None
        if vectors is not None:
            vm = mat(vectors[0], vectors[1], columns=k, rows=self.cfg.n)
        self._cb_error = None
        st = getattr(lib(), _entry)(self.h, er, ei, rs, C.byref(vm) if vm else None)
        if st == ERR_CALLBACK and self._cb_error is not None:
            raise OapbError(st, _entry) from self._cb_error
        if not (st == OK or (allow_not_converged and st == NOT_CONVERGED)):
            raise OapbError(st, _entry)
        return [complex(er[i], ei[i]) for i in range(k)], list(rs), st

    def resume(self, vectors=None, allow_not_converged=False):
        """Continue from the loaded (or last) factorization (oapb_arnoldi_resume)."""
        return self.solve(vectors, allow_not_converged, _entry="oapb_arnoldi_resume")

    def set_gram_operator(self, X):
        """Implicit Gram operator A = X X^T of a (n, pixels) FP32 device tensor."""
        assert X.dtype.is_floating_point and X.element_size() == 4 and X.is_contiguous() and X.is_cuda
        self._ops = (X,)
        check(lib().oapb_arnoldi_set_gram_operator(self.h, C.c_void_p(X.data_ptr()), X.shape[0], X.shape[1]),
              "oapb_arnoldi_set_gram_operator")

    def set_gram_operator_host(self, X, block_cols, resident_bytes=0):
        """Implicit Gram operator A = X X^T with X (n, pixels) FP32 in HOST
        memory (a C-contiguous numpy array or a pinned CPU tensor), applied by
        column blocks of block_cols pixels; the blocks that fit resident_bytes
        stay on the device, the rest stream on every application."""
        import numpy as np
        if hasattr(X, "data_ptr"):
            assert X.dtype.is_floating_point and X.element_size() == 4 and X.is_contiguous() and not X.is_cuda
            ptr, rows, cols = X.data_ptr(), X.shape[0], X.shape[1]
        else:
            assert X.dtype == np.float32 and X.flags.c_contiguous
            ptr, rows, cols = X.ctypes.data, X.shape[0], X.shape[1]
        self._ops = (X,)
        check(lib().oapb_arnoldi_set_gram_operator_host(self.h, C.c_void_p(ptr), rows, cols, block_cols,
                                                        int(resident_bytes)),
              "oapb_arnoldi_set_gram_operator_host")

    def gram_stream_info(self):
        """(blocks, resident blocks, host-to-device bytes streamed so far)."""
        nb, nr, by = C.c_uint32(), C.c_uint32(), C.c_uint64()
        check(lib().oapb_arnoldi_gram_stream_info(self.h, C.byref(nb), C.byref(nr), C.byref(by)),
              "oapb_arnoldi_gram_stream_info")
        return nb.value, nr.value, by.value

    def save(self, path):
        check(lib().oapb_arnoldi_save(self.h, str(path).encode()), "oapb_arnoldi_save")

    def load(self, path):
        check(lib().oapb_arnoldi_load(self.h, str(path).encode()), "oapb_arnoldi_load")

    def solve_host(self, are, aim=None, vectors=False):
        """Dense solve from host FP64 arrays (numpy, C-contiguous)."""
        import numpy as np
        k, n = self.cfg.wanted, self.cfg.n
        er, ei, rs = (C.c_double * k)(), (C.c_double * k)(), (C.c_double * k)()
        vr = np.zeros((n, k)) if vectors else None
        vi = np.zeros((n, k)) if (vectors and aim is not None) else None
        p = lambda a: C.c_void_p(a.ctypes.data) if a is not None else None
        st = lib().oapb_arnoldi_solve_host(self.h, p(are), p(aim), er, ei, rs, p(vr), p(vi))
        if st not in (OK, NOT_CONVERGED):
            raise OapbError(st, "oapb_arnoldi_solve_host")
        out = [complex(er[i], ei[i]) for i in range(k)], list(rs), st
        if vectors:
            return out + (vr if vi is None else vr + 1j * vi,)
        return out

    def apply_block(self, xre, xim=None, precision=PREC_FP64):
        """W = A X for X given as (b, n) device FP64 tensors."""
        import torch
        b = xre.shape[0]
        wre = torch.empty_like(xre)
        wim = torch.empty_like(xim) if xim is not None else None
        p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
        check(lib().oapb_arnoldi_apply_block(self.h, p(xre), p(xim), b, p(wre), p(wim), precision),
              "oapb_arnoldi_apply_block")
        return wre, wim

    def set_profile(self, on):
        """Per-launch CUDA-event timing of the operator passes on / off."""
        check(lib().oapb_arnoldi_set_profile(self.h, int(bool(on))), "oapb_arnoldi_set_profile")

    def trace(self):
        """Convergence checks of the last solve: (phase, iteration, passes,
        bf16_passes, residual) tuples (phase 1: FP32-class subspace
        iteration, 2: FP64 subspace iteration, 3: FP64-anchored refinement)."""
        cnt = C.c_uint32()
        check(lib().oapb_arnoldi_get_trace(self.h, None, 0, C.byref(cnt)), "oapb_arnoldi_get_trace")
        recs = (TraceRec * max(cnt.value, 1))()
        check(lib().oapb_arnoldi_get_trace(self.h, recs, cnt.value, C.byref(cnt)), "oapb_arnoldi_get_trace")
        return [(r.phase, r.iteration, r.passes, r.bf16_passes, r.residual) for r in recs[:cnt.value]]

    def stats(self):
        s = Stats()
        check(lib().oapb_arnoldi_get_stats(self.h, C.byref(s)), "oapb_arnoldi_get_stats")
        return {f: (list(getattr(s, f)) if isinstance(getattr(s, f), C.Array) else getattr(s, f))
                for f, _ in Stats._fields_}

    def test_outcome(self, index):
        out = C.c_double()
        check(lib().oapb_arnoldi_test_outcome(self.h, index, C.byref(out)),
              "oapb_arnoldi_test_outcome")
        return out.value


def selftest_bounded_wait(limit_us, arrive=False, stream=None):
    """Run the bounded device-side wait self-test (oapb_selftest_bounded_wait):
    returns (status, timed_out).  arrive=False lets the wait run out."""
    out = C.c_int32(-1)
    st = lib().oapb_selftest_bounded_wait(int(limit_us), int(bool(arrive)), C.byref(out), _stream(stream))
    return st, out.value


def start_vector(n, seed, is_complex=False):
    """Host restatement of the library's seeded U[-1, 1) start vector
    (splitmix64 of seed * 0x100000001B3 + i), for comparing with the oracle."""
    import numpy as np
    M = (1 << 64) - 1

    def uni(seed_, i):
        z = (seed_ * 0x100000001B3 + i) & M
        z = (z + 0x9E3779B97F4A7C15) & M
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        z = z ^ (z >> 31)
        return (z >> 11) * (2.0 / 9007199254740992.0) - 1.0

    re = np.array([uni(seed, i) for i in range(n)])
    if not is_complex:
        return re
    s2 = seed ^ 0x5851F42D4C957F2D
    im = np.array([uni(s2, i) for i in range(n)])
    return re + 1j * im


def solve_batched(mats, wanted, hdim=24, sort="LM", tolerance=1e-10, max_restarts=300,
                  rho=1.0 / 3.14, seed=1, vectors=None, stream=None, autotune=True):
    """Batched solve of independent problems.  mats: list of (re, im) device
    tensors (im None for real problems); vectors: optional list of (vre, vim)
    device tensors of shape (n, wanted); autotune: True (tune the launch
    variant once per shape), False (default variant) or 2 + v (variant v).  Returns (eigenvalues [count x
    wanted] complex, residuals, status per problem, stats dict, rc)."""
    import numpy as np
    L = lib()
    cfg = Config()
    L.oapb_arnoldi_config_default(C.byref(cfg))
    cfg.hdim, cfg.wanted = hdim, wanted
    cfg.sort = SORT[sort] if isinstance(sort, str) else int(sort)
    cfg.tolerance, cfg.max_restarts, cfg.rho, cfg.seed = tolerance, max_restarts, rho, seed
    cfg.autotune = int(autotune)
    cnt = len(mats)
    probs = (BatchProblem * cnt)()
    for i, (re, im) in enumerate(mats):
        probs[i].n = re.shape[0]
        probs[i].re = re.data_ptr()
        probs[i].im = im.data_ptr() if im is not None else None
        if vectors is not None:
            vr, vi = vectors[i]
            probs[i].eigvec_re = vr.data_ptr()
            probs[i].eigvec_im = vi.data_ptr() if vi is not None else None
    er = np.zeros((cnt, wanted))
    ei = np.zeros((cnt, wanted))
    rs = np.zeros((cnt, wanted))
    st = np.zeros(cnt, dtype=np.int32)
    stats = BatchStats()
    P = lambda a, t=C.c_double: a.ctypes.data_as(C.POINTER(t))
    rc = L.oapb_arnoldi_solve_batched(C.byref(cfg), probs, cnt, P(er), P(ei), P(rs),
                                      P(st, C.c_int32), C.byref(stats), _stream(stream))
    if rc not in (OK, NOT_CONVERGED):
        raise OapbError(rc, "oapb_arnoldi_solve_batched")
    return (er + 1j * ei, rs, st, {f: getattr(stats, f) for f, _ in BatchStats._fields_}, rc)


def gram_build(X, fp64=False, stream=None):
    """A = X X^T (split-BF16 tensor-core GEMM) for a row-major FP32 CUDA
    tensor X (rows x cols).  Returns (A float32, A64 float64 or None)."""
    import torch
    assert X.is_cuda and X.dtype == torch.float32 and X.is_contiguous()
    rows, cols = X.shape
    A = torch.empty((rows, rows), dtype=torch.float32, device=X.device)
    A64 = torch.empty((rows, rows), dtype=torch.float64, device=X.device) if fp64 else None
    check(lib().oapb_gram_build(C.c_void_p(X.data_ptr()), rows, cols, C.c_void_p(A.data_ptr()),
                                C.c_void_p(A64.data_ptr()) if fp64 else None, _stream(stream)),
          "oapb_gram_build")
    return A, A64


def mat_write(path, re, im=None, stream=None):
    """Write device FP64 planes (2-D torch tensors, rows x columns) as a matrix
    file in the reference's format (oapb_mat_write)."""
    m = mat(re, im)
    check(lib().oapb_mat_write(str(path).encode(), C.byref(m), _stream(stream)), "oapb_mat_write")


def mat_read_info(path):
    """(columns, rows, has_re, has_im) of the first matrix of a file."""
    c, r, hr, hi = C.c_uint32(), C.c_uint32(), C.c_int32(), C.c_int32()
    check(lib().oapb_mat_read_info(str(path).encode(), C.byref(c), C.byref(r), C.byref(hr), C.byref(hi)),
          "oapb_mat_read_info")
    return c.value, r.value, bool(hr.value), bool(hi.value)


def mat_read(path, device="cuda", stream=None):
    """Read a matrix file into new device FP64 tensors (re, im or None)."""
    import torch
    c, r, hr, hi = mat_read_info(path)
    re = torch.empty(r, c, dtype=torch.float64, device=device)
    im = torch.empty(r, c, dtype=torch.float64, device=device) if hi else None
    m = mat(re, im)
    check(lib().oapb_mat_read(str(path).encode(), C.byref(m), _stream(stream)), "oapb_mat_read")
    return re, im


def images_to_matrix(rgb, stream=None):
    """(count, pixels, 3) uint8 RGB images (numpy on the host or a torch
    device tensor) -> X (count, pixels) FP32 device tensor, each pixel
    (r << 16 | g << 8 | b) / 0xFFFFFF (oapb_images_to_matrix)."""
    import numpy as np
    import torch
    count, pixels = int(rgb.shape[0]), int(rgb.shape[1])
    X = torch.empty(count, pixels, dtype=torch.float32, device="cuda")
    if isinstance(rgb, np.ndarray):
        a = np.ascontiguousarray(rgb, dtype=np.uint8)
        ptr, host = C.c_void_p(a.ctypes.data), 1
    else:
        a = rgb.contiguous()
        ptr, host = C.c_void_p(a.data_ptr()), 0
    check(lib().oapb_images_to_matrix(ptr, host, count, pixels, C.c_void_p(X.data_ptr()), _stream(stream)),
          "oapb_images_to_matrix")
    return X
