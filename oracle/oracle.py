"""Test infrastructure (oracle): ctypes bindings for the CPU checkers.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module; the product path never does.

Two checkers live behind it:

* ``Port``  -- lib/liboracle_fp{64,32}.so, the plain-C restatement of the
  reference's eval_RHS_swe and RK4 stage combine (swe_oracle.c; reference
  swe_code/main/rk4_rbffd_swe.c:30-362) on the canonical node-major layout.
* ``Ref``   -- _ref/libswe_ref_<prec>_<layout>.so, the reference mini-app's own
  sources compiled from where they lie (Makefile) with ref_harness.c, which
  replays main.c's initialisation and exposes the reference's RK_substep and
  eval_RHS_swe.  It exists only where the reference was present at build time
  (and on machines the built files were shipped to).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "lib")
REF_DIR = os.path.join(HERE, "_ref")
SHIPPED_INPUT = os.path.join(REF_DIR, "icos2562_tc5_input.bin")
LAYOUTS = ("default", "cfdl", "sfdl", "cfdl_sfdl")
LAYOUT_FLAGS = {"default": 0, "cfdl": 1, "sfdl": 2, "cfdl_sfdl": 3}


def usable_cpus() -> dict:
    """The CPUs this process may really use: its affinity set, capped by a cgroup CPU
    quota (cgroup v2 cpu.max, else v1 cfs_quota_us / cfs_period_us) rounded down, at
    least 1.  os.cpu_count() counts the machine's CPUs and ignores both, and a static
    OpenMP schedule over more threads than the quota allows waits at every barrier
    for threads that are not running."""
    try:
        affinity = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        affinity = os.cpu_count() or 1
    quota = None
    try:
        q, period = open("/sys/fs/cgroup/cpu.max").read().split()[:2]
        if q != "max":
            quota = int(q) / int(period)
    except (OSError, ValueError):
        try:
            q = int(open("/sys/fs/cgroup/cpu/cpu.cfs_quota_us").read())
            period = int(open("/sys/fs/cgroup/cpu/cpu.cfs_period_us").read())
            if q > 0:
                quota = q / period
        except (OSError, ValueError):
            pass
    threads = affinity if quota is None else max(1, min(affinity, int(quota)))
    model = ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"threads": threads, "affinity": affinity, "cpu_count": os.cpu_count(),
            "cgroup_quota_cpus": quota, "model": model}


def set_thread_count(n: int) -> None:
    """OpenMP threads for later parallel regions of the calling thread (libgomp, which
    the oracle and reference libraries link)."""
    ctypes.CDLL("libgomp.so.1").omp_set_num_threads(int(n))


def build(with_reference: bool | None = None) -> None:
    """Build the port (always) and the reference libraries (when the reference is present)."""
    # the reference project root: SWE_REFERENCE_DIR, else a checkout named `reference`
    # beside this repository
    ref_root = os.environ.get("SWE_REFERENCE_DIR",
                              os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))
    if with_reference is None:
        with_reference = os.path.isdir(os.path.join(ref_root, "swe_code"))
    targets = ["port"] + (["ref"] if with_reference else [])
    lib = os.path.join(os.path.dirname(HERE), "rbf-fd-swe_b200", "lib", "libswe_b200.so")
    if with_reference and os.path.exists(lib):
        targets.append("host")          # the reference's main program driving the library
    subprocess.run(["make", "-s", "-C", HERE, f"REF_DIR={ref_root}", "-j8", *targets], check=True)


def reference_available(prec: str = "fp64", layout: str = "cfdl") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libswe_ref_{prec}_{layout}.so"))


class _Grid(ctypes.Structure):
    """Mirror of OracleGrid in swe_oracle.c."""

    _fields_ = [("n", ctypes.c_int), ("nnbr", ctypes.c_int), ("stride", ctypes.c_int),
                ("gh0", ctypes.c_double), ("dt", ctypes.c_double)] + \
               [(name, ctypes.c_void_p) for name in
                ("idx", "Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm")]


class _Grid32(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("nnbr", ctypes.c_int), ("stride", ctypes.c_int),
                ("gh0", ctypes.c_float), ("dt", ctypes.c_float)] + \
               [(name, ctypes.c_void_p) for name in
                ("idx", "Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm")]


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Port:
    """The C restatement, bound to one model in canonical layout.

    ``model`` is a swe_b200.swe_input.SweModel (or any object with the same
    fields): FP64 arrays node-major, idx 0-based.  ``prec`` is "fp64" or
    "fp32"; in fp32 every array is rounded to float first, as the reference's
    reader does (input.c:189-332 casts fType_Input to fType).
    """

    def __init__(self, model, prec: str = "fp64"):
        self.prec = prec
        self.dtype = np.float64 if prec == "fp64" else np.float32
        path = os.path.join(LIB_DIR, f"liboracle_{prec}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle port`")
        self.lib = ctypes.CDLL(path)
        dt = self.dtype
        self.n, self.nnbr = int(model.N), int(model.Nnbr)
        self._keep = {
            "idx": np.ascontiguousarray(model.idx, dtype=np.int32),
            **{k: np.ascontiguousarray(getattr(model, k), dtype=dt)
               for k in ("Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm")},
        }
        G = _Grid if prec == "fp64" else _Grid32
        self.grid = G(self.n, self.nnbr, self.nnbr, float(model.gh0), float(model.dt),
                      *[_ptr(self._keep[k]) for k in
                        ("idx", "Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm")])
        self.lib.oracle_eval_rhs.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        self.lib.oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        self.lib.oracle_rk_substep.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_int]
        self.lib.oracle_invariants.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]

    def eval_rhs(self, K: np.ndarray) -> np.ndarray:
        K = np.ascontiguousarray(K, dtype=self.dtype).reshape(-1, 4)
        F = np.zeros((self.n, 4), dtype=self.dtype)
        self.lib.oracle_eval_rhs(ctypes.byref(self.grid), _ptr(K), _ptr(F))
        return F

    def run(self, H: np.ndarray, nsteps: int) -> np.ndarray:
        H = np.array(H, dtype=self.dtype, order="C").reshape(self.n, 4)
        self.lib.oracle_run(ctypes.byref(self.grid), _ptr(H), int(nsteps))
        return H

    def rk_substep(self, H: np.ndarray, K: np.ndarray, F: np.ndarray, D: np.ndarray, substep_id: int) -> None:
        """RK_substep (rk4_rbffd_swe.c:30-72) on [n][4] arrays of this precision, in place."""
        for a in (H, K, F, D):
            assert a.dtype == self.dtype and a.flags.c_contiguous and a.size == 4 * self.n
        self.lib.oracle_rk_substep(ctypes.byref(self.grid), _ptr(H), _ptr(K), _ptr(F), _ptr(D), int(substep_id))

    def invariants(self, H: np.ndarray) -> np.ndarray:
        """FP64 (mass, energy) per member for H of shape [members, n, 4] or [n, 4]."""
        H = np.ascontiguousarray(H, dtype=self.dtype).reshape(-1, self.n, 4)
        out = np.zeros((H.shape[0], 2), dtype=np.float64)
        self.lib.oracle_invariants(ctypes.byref(self.grid), _ptr(H), H.shape[0], _ptr(out))
        return out


class Ref:
    """The reference's own C code (one layout/precision build) via ref_harness.c."""

    def __init__(self, path_input: str, prec: str = "fp64", layout: str = "cfdl", use_rcm: int = 1):
        so = os.path.join(REF_DIR, f"libswe_ref_{prec}_{layout}.so")
        if not os.path.exists(so):
            raise FileNotFoundError(f"{so} missing: the reference was not built here")
        if not os.path.exists(path_input):
            # the reference's reader exit()s on a missing file (input.c:8); check first
            raise FileNotFoundError(path_input)
        self.prec, self.layout = prec, layout
        self.dtype = np.float64 if prec == "fp64" else np.float32
        lib = ctypes.CDLL(so)
        self.lib = lib
        lib.refh_load.argtypes = [ctypes.c_char_p, ctypes.c_int]
        lib.refh_info.argtypes = [ctypes.c_void_p]
        for name in ("refh_psmd", "refh_H_init", "refh_H_100", "refh_mapping"):
            getattr(lib, name).restype = ctypes.c_void_p
        lib.refh_array.restype = ctypes.c_void_p
        lib.refh_array.argtypes = [ctypes.c_char_p]
        lib.refh_eval_rhs.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.refh_rk_substep.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int]
        lib.refh_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        lib.refh_run.restype = ctypes.c_double
        lib.refh_verify.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        lib.refh_tolerance.restype = ctypes.c_double
        lib.refh_gh0.restype = ctypes.c_double
        lib.refh_dt.restype = ctypes.c_double
        if lib.refh_load(path_input.encode(), int(use_rcm)) != 0:
            raise RuntimeError("refh_load failed")
        info = (ctypes.c_int * 9)()
        lib.refh_info(info)
        (self.patch_size, self.compute_size, self.Nnbr, self.padded_Nnbr, fsize,
         self.layout_flags, self.simd_length, self.compute_pid_s, self.Nnodes) = list(info)
        assert fsize == np.dtype(self.dtype).itemsize
        self.tolerance = lib.refh_tolerance()

    def psmd_ptr(self) -> int:
        return self.lib.refh_psmd()

    def _view(self, addr: int, count: int, dtype) -> np.ndarray:
        buf = (ctypes.c_char * (count * np.dtype(dtype).itemsize)).from_address(addr)
        return np.frombuffer(buf, dtype=dtype).copy()

    def H_init(self) -> np.ndarray:
        return self._view(self.lib.refh_H_init(), self.patch_size * 4, self.dtype)

    def H_100(self) -> np.ndarray:
        return self._view(self.lib.refh_H_100(), self.patch_size * 4, self.dtype)

    def mapping(self) -> np.ndarray:
        return self._view(self.lib.refh_mapping(), self.Nnodes, np.int32)

    def array(self, name: str) -> np.ndarray:
        n = self.compute_size
        counts = {"x": n, "y": n, "z": n, "f": n, "ghm": n,
                  "p_u": 3 * n, "p_v": 3 * n, "p_w": 3 * n, "gradghm": 3 * n,
                  "idx": n * self.padded_Nnbr, "Dx": n * self.padded_Nnbr, "Dy": n * self.padded_Nnbr,
                  "Dz": n * self.padded_Nnbr, "L": n * self.padded_Nnbr}
        dt = np.int32 if name == "idx" else self.dtype
        return self._view(self.lib.refh_array(name.encode()), counts[name], dt)

    def eval_rhs(self, K: np.ndarray) -> np.ndarray:
        K = np.ascontiguousarray(K, dtype=self.dtype)
        assert K.size == self.patch_size * 4
        F = np.zeros(self.compute_size * 4, dtype=self.dtype)
        self.lib.refh_eval_rhs(_ptr(K), _ptr(F))
        return F

    def run(self, H: np.ndarray, nsteps: int):
        """nsteps RK4 steps from H (reference layout); returns (H, loop_seconds, eval_rhs_seconds)."""
        H = np.array(H, dtype=self.dtype, order="C")
        t_rhs = ctypes.c_double(0.0)
        t = self.lib.refh_run(_ptr(H), int(nsteps), ctypes.byref(t_rhs))
        return H, t, t_rhs.value

    def verify(self, H: np.ndarray):
        """(count of |H - H_100| > TOLERANCE, max abs error): main.c verify_output."""
        H = np.ascontiguousarray(H, dtype=self.dtype)
        mx = ctypes.c_double(0.0)
        c = self.lib.refh_verify(_ptr(H), ctypes.byref(mx))
        return int(c), mx.value

    # -- layout helpers (reference layout <-> canonical [patch_size, 4]) ---------------
    def state_to_canonical(self, H: np.ndarray) -> np.ndarray:
        """Reference-layout state -> [patch_size, 4] (SVM_LIN_ID, swe_config.h:50-54)."""
        S = self.simd_length
        H = np.asarray(H).reshape(-1)
        if self.layout_flags & 1:
            return H.reshape(-1, 4).copy()
        return H.reshape(-1, 4, S).transpose(0, 2, 1).reshape(-1, 4).copy()

    def state_from_canonical(self, C: np.ndarray) -> np.ndarray:
        S = self.simd_length
        C = np.asarray(C, dtype=self.dtype).reshape(-1, 4)
        if self.layout_flags & 1:
            return C.reshape(-1).copy()
        return C.reshape(-1, S, 4).transpose(0, 2, 1).reshape(-1).copy()
