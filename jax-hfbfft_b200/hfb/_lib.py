"""ctypes binding of libhfb.so (include/hfb.h).

The library is built in-tree by ``jax-hfbfft_b200/build.py``.  Loading fails
loudly when it is missing: there is no CPU fallback.
"""
import ctypes as C
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhfb.so")

HFB_OK = 0
HFB_ERR_CUDA = 3
HFB_ERR_NONFINITE = 6
HFB_ERR_TIMEOUT = 8
HFB_F64 = 0
HFB_F32 = 1
STATUS = {0: "ok", 1: "invalid argument", 2: "unsupported grid", 3: "CUDA error",
          4: "BCS particle number not bracketed on [-100, 100]", 5: "iteration limit reached",
          6: "non-finite value", 7: "device allocation failed", 8: "a bounded device wait ran out"}
ENERGY_KEYS = ("ehft", "ehf0", "ehf1", "ehf2", "ehf3", "ehfls", "ehflsodd", "ehfc", "ecorc", "ehfint",
               "e3corr", "e_zpe", "ehf", "tke", "ehfCrho0", "ehfCrho1", "ehfCdrho0", "ehfCdrho1",
               "ehfCtau0", "ehfCtau1", "ehfCdJ0", "ehfCdJ1", "ehfCj0", "ehfCj1")
HFB_NE = len(ENERGY_KEYS)

vp = C.c_void_p
dp = C.c_void_p   # device double* passed as an address


class HfbForce(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("b0", "b0p", "b1", "b1p", "b2", "b2p", "b3", "b3p", "b4", "b4p",
                                          "power", "slate")] + \
               [("h2m", C.c_double * 2), ("h2ma", C.c_double), ("v0neut", C.c_double), ("v0prot", C.c_double),
                ("rho0pr", C.c_double)] + \
               [(n, C.c_double) for n in ("Crho0", "Crho1", "Crho0D", "Crho1D", "Cdrho0", "Cdrho1", "Ctau0",
                                          "Ctau1", "CdJ0", "CdJ1")] + \
               [("ipair", C.c_int), ("ex", C.c_int), ("zpe", C.c_int), ("pad_", C.c_int)]


class GrstepArgs(C.Structure):
    _fields_ = [("nst", C.c_int), ("nneut", C.c_int), ("tbcs", C.c_int), ("use_lagrange", C.c_int),
                ("do_fluct", C.c_int), ("pad_", C.c_int),
                ("x0dmp", C.c_double), ("e0dmp", C.c_double), ("h2ma", C.c_double), ("wxyz", C.c_double),
                ("pot", vp), ("v_pair", vp), ("psi", vp), ("hampsi", vp), ("hmfpsi", vp), ("delpsi", vp),
                ("lagrange", vp), ("wocc", vp), ("wguv", vp), ("pairwg", vp), ("wstates", vp),
                ("sp_energy", vp), ("sp_efluct1", vp), ("sp_efluct2", vp), ("sums", vp), ("x0dmp_dev", vp)]


class DiagArgs(C.Structure):
    _fields_ = [("npsi", C.c_int * 2), ("nmax", C.c_int), ("diagonalize", C.c_int), ("construct", C.c_int),
                ("ipair", C.c_int), ("tbcs", C.c_int), ("pad_", C.c_int), ("wxyz", C.c_double),
                ("psi", vp), ("psi_out", vp), ("hampsi", vp), ("hmfpsi", vp), ("lagrange", vp), ("v_pair", vp),
                ("wocc", vp), ("wguv", vp), ("pairwg", vp), ("wstates", vp), ("sp_norm", vp), ("sp_energy", vp),
                ("deltaf", vp), ("hmatrix", vp), ("gapmatrix", vp), ("symcond", vp), ("lambda_save", vp),
                ("efluct", vp)]


class PairArgs(C.Structure):
    _fields_ = [("npsi", C.c_int * 2), ("nneut", C.c_int), ("nprot", C.c_int), ("use_const_gap", C.c_int),
                ("pad_", C.c_int), ("const_gap", C.c_double), ("pair_cutoff", C.c_double * 2),
                ("state_cutoff", C.c_double * 2), ("softcut_range", C.c_double),
                ("sp_energy", vp), ("deltaf", vp), ("wocc", vp), ("wguv", vp), ("pairwg", vp), ("wstates", vp),
                ("out", vp)]


class NaturalArgs(C.Structure):
    _fields_ = [("nst", C.c_int), ("ld", C.c_int), ("iq", C.c_int), ("start", C.c_int), ("ipair", C.c_int),
                ("pad_", C.c_int), ("delstepbas", C.c_double), ("e0bas", C.c_double),
                ("hmatrix", vp), ("gapmatrix", vp), ("symcond", vp), ("lambda_save", vp), ("sp_energy", vp),
                ("deltaf", vp), ("wocc", vp), ("wguv", vp), ("pairwg", vp), ("wstates", vp)]


# symbol -> argument types (restype int unless noted)
_PROTOS = {
    "hfb_ctx_create": [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                       C.POINTER(vp)],
    "hfb_ctx_destroy": [vp],
    "hfb_device_status": [vp, vp, C.POINTER(C.c_int)],
    "hfb_set_wait_limit": [vp, C.c_longlong],
    "hfb_arm_timeout_probe": [vp],
    "hfb_set_hpsi_kernel": [vp, C.c_int],
    "hfb_cderv": [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp],
    "hfb_laplace": [vp, C.c_int, C.c_int, vp, vp, vp, C.c_double, C.c_double, C.c_double, vp, vp],
    "hfb_hpsi": [vp, C.c_int, vp, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp, vp],
    "hfb_skyrme": [vp, C.POINTER(HfbForce), C.c_int] + [vp] * 6 + [vp] * 8 + [vp, vp, C.c_int, vp, vp],
    "hfb_poisson": [vp, vp, vp, vp],
    "hfb_poisson_noalloc": [vp, vp, vp, vp],
    "hfb_add_density": [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, C.c_double] + [vp] * 6 +
                       [C.POINTER(C.c_double), vp, vp],
    "hfb_sp_kinetic": [vp, C.c_int, C.c_int, C.c_int, vp, C.POINTER(C.c_double), vp, vp],
    "hfb_harmosc": [vp, C.c_int, C.c_int, vp, C.c_double, C.c_double, C.c_double, vp, vp],
    "hfb_grstep": [vp, C.c_int, C.POINTER(GrstepArgs), vp],
    "hfb_diagstep": [vp, C.c_int, C.POINTER(DiagArgs), vp],
    "hfb_gram": [vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, vp, vp],
    "hfb_eigh": [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp],
    "hfb_eigh_near_diagonal": [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp],
    "hfb_pair": [vp, C.POINTER(PairArgs), vp],
    "hfb_lastdiag": [vp, C.c_int, C.c_int, vp, vp, vp, vp, C.c_int, vp, vp, vp],
    "hfb_natural_begin": [vp, C.POINTER(NaturalArgs), vp],
    "hfb_step_control": [vp, vp, vp, vp, vp, vp, C.c_int, vp],
    "hfb_state_dot": [vp, C.c_int, C.c_int, vp, vp, vp, vp],
    "hfb_state_axpby": [vp, C.c_int, C.c_int, C.c_double, vp, C.c_double, vp, vp],
    "hfb_state_mul_field": [vp, C.c_int, C.c_int, vp, vp, vp, vp],
    "hfb_state_project": [vp, C.c_int, C.c_int, vp, C.c_int, vp, vp],
    "hfb_state_axpby_diag": [vp, C.c_int, C.c_int, vp, vp, C.c_double, vp, vp],
    "hfb_rms_field": [vp, C.POINTER(C.c_double), C.c_double, C.c_double, vp, vp],
    "hfb_nyquist_pair": [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp],
    "hfb_nyquist_apply": [vp, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp],
    "hfb_natural_step": [vp, C.POINTER(NaturalArgs), C.c_int, vp],
    "hfb_natural_symcond": [vp, C.POINTER(NaturalArgs), vp],
    "hfb_natural_end": [vp, C.c_int, C.POINTER(NaturalArgs), vp, vp, vp, vp],
    "hfb_energies": [vp, C.POINTER(HfbForce), C.c_int, C.c_double] + [vp] * 6 + [vp, vp, vp],
    "hfb_sum_energy": [vp, C.c_int] + [vp] * 6 + [vp, vp],
    "hfb_energy_grad": [vp, C.POINTER(HfbForce)] + [vp] * 5 + [vp, vp],
    "hfb_rms": [vp, vp, vp, vp],
    "hfb_observables": [vp, vp, vp, C.c_double, C.c_double, vp, vp],
    "hfb_sp_properties": [vp, C.c_int, C.c_int, vp, C.POINTER(C.c_double), vp, vp, vp, vp],
    "hfb_constraint_fields": [vp, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, vp, vp],
    "hfb_constraint_moments": [vp, C.c_int, vp, vp, vp, vp],
    "hfb_constraint_potential": [vp, C.c_int, C.c_int, vp, C.POINTER(C.c_double), vp, vp, vp],
    "hfb_constraint_correct": [vp, C.c_int, C.c_int, C.c_int, vp, C.POINTER(C.c_double), vp, vp, vp, vp],
}
SYMBOLS = tuple(_PROTOS) + ("hfb_status_string", "hfb_launch_count", "hfb_last_cuda_error")

_lib = None


def load():
    """Load libhfb.so and declare every prototype; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libhfb.so not found at {LIB_PATH}; build it with jax-hfbfft_b200/build.py")
    lib = C.CDLL(LIB_PATH)
    for name, args in _PROTOS.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = C.c_int
    lib.hfb_status_string.argtypes = [C.c_int]
    lib.hfb_status_string.restype = C.c_char_p
    lib.hfb_launch_count.argtypes = []
    lib.hfb_launch_count.restype = C.c_ulonglong
    lib.hfb_last_cuda_error.argtypes = [C.POINTER(C.c_int)]
    lib.hfb_last_cuda_error.restype = C.c_char_p
    _lib = lib
    return lib


class HfbError(RuntimeError):
    def __init__(self, fn, code, detail=""):
        super().__init__(f"{fn}: {STATUS.get(code, 'unknown status')} (status {code}){detail}")
        self.code = code


def call(name, *args):
    """Call a library function and raise HfbError on a non-zero status."""
    r = getattr(load(), name)(*args)
    if r != HFB_OK:
        detail = ""
        if r == HFB_ERR_CUDA:
            e = C.c_int(0)
            msg = load().hfb_last_cuda_error(C.byref(e)).decode()
            detail = f": cudaError {e.value} ({msg})"
        raise HfbError(name, r, detail)
    return r


def ptr(t):
    """Device address of a CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


def launch_count():
    """Kernels launched by libhfb in this process so far."""
    return int(load().hfb_launch_count())


def stream_ptr():
    return torch.cuda.current_stream().cuda_stream


def prec_of(t):
    if t.dtype == torch.complex128:
        return HFB_F64
    if t.dtype == torch.complex64:
        return HFB_F32
    raise TypeError(f"unsupported state dtype {t.dtype}")


class Context:
    """Owns one hfb_ctx_t (grid, derivative matrices, Coulomb kernel, scratch)."""

    def __init__(self, n, d, periodic=False, nstmax=0):
        lib = load()
        if not torch.cuda.is_available():
            raise RuntimeError("hfb needs a CUDA device")
        torch.cuda.init()
        h = vp()
        call("hfb_ctx_create", n[0], n[1], n[2], float(d[0]), float(d[1]), float(d[2]), int(bool(periodic)),
             int(nstmax), C.byref(h))
        self.handle = h
        self._lib = lib

    def __del__(self):
        try:
            if self.handle:
                self._lib.hfb_ctx_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def device_status(self):
        s = C.c_int(0)
        call("hfb_device_status", self.handle, stream_ptr(), C.byref(s))
        return s.value

    def check(self, what="device"):
        s = self.device_status()
        if s != HFB_OK:
            raise HfbError(what, s)
