"""ctypes binding of the C ABI in include/swe_b200.h (lib/libswe_b200.so).

This is the Python face of the drop-in boundary: the same entry points a C
host (the reference's main.c with its SWE_USE_CUDA branch) calls.  Arrays are
numpy host buffers in the caller's layout.  There is no fallback: if the
shared library is missing or a call fails, an exception says so.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# SWE_B200_LIB names another build of the library (a test run against a variant build)
LIB_PATH = os.environ.get("SWE_B200_LIB") or os.path.join(PKG_DIR, "lib", "libswe_b200.so")
HEADER = os.path.join(os.path.dirname(PKG_DIR), "include", "swe_b200.h")

SWE_LAYOUT_CFDL = 1
SWE_LAYOUT_SFDL = 2
STATUS = {0: "SWE_OK", 1: "SWE_ERR_ARG", 2: "SWE_ERR_STATE", 3: "SWE_ERR_CUDA", 4: "SWE_ERR_NOMEM",
          5: "SWE_ERR_INDEX", 6: "SWE_ERR_TIMEOUT", 7: "SWE_ERR_NONFINITE", 8: "SWE_ERR_CANCELLED"}



def _header_define(name: str) -> int:
    m = re.search(r"#define\s+%s\s+\((\d+)u\s*<<\s*(\d+)\)" % name, open(HEADER).read())
    if not m:
        raise RuntimeError(f"{name} not found in {HEADER}")
    return int(m.group(1)) << int(m.group(2))


# bytes of the static device array swe_cuda_step_noalloc keeps K and D in
NOALLOC_SCRATCH_BYTES = _header_define("SWE_NOALLOC_SCRATCH_BYTES")

_lib = None


class SweError(RuntimeError):
    def __init__(self, fn: str, status: int, msg: str):
        super().__init__(f"{fn} -> {STATUS.get(status, status)}: {msg}")
        self.status = status


def declared_symbols() -> list[str]:
    """Every function name include/swe_b200.h declares with C linkage."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    body = text.split('extern "C" {', 1)[1].split("#ifdef __cplusplus\n}", 1)[0]
    return sorted(set(re.findall(r"\b(swe_\w+)\s*\(", body)))


def load() -> ctypes.CDLL:
    """Load lib/libswe_b200.so (once); raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: the sm_100a library was not built "
                           f"(run __graft_entry__.build() or make -C {PKG_DIR})")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    lib.swe_cuda_last_error.restype = ctypes.c_char_p
    lib.swe_b200_kernel_launches.restype = ctypes.c_longlong
    lib.swe_cuda_init.argtypes = [i, i, i, i, i, i, i, i, d, d] + [vp] * 14
    for name in ("swe_cuda_set_state", "swe_cuda_get_state", "swe_cuda_last_timings", "swe_cuda_invariants"):
        getattr(lib, name).argtypes = [vp]
    lib.swe_cuda_eval_rhs.argtypes = [vp, vp]
    lib.swe_cuda_rk_substep.argtypes = [i]
    lib.swe_cuda_step.argtypes = [i]
    lib.swe_cuda_set_timing.argtypes = [i]
    lib.swe_cuda_stream.restype = vp
    lib.swe_cuda_select_kernel.argtypes = [i]
    lib.swe_cuda_kernel_info.argtypes = [vp]
    lib.swe_cuda_set_index_width.argtypes = [i]
    lib.swe_hist_open.argtypes = [ctypes.c_char_p, i]
    lib.swe_gen_stencils.argtypes = [i, i, vp, vp]
    lib.swe_selftest_wait_timeout.argtypes = [d, vp]
    lib.swe_gen_weights.argtypes = [i, i, vp, vp, vp]
    lib.swe_hist_stats.argtypes = [vp]
    lib.swe_ens_init.argtypes = [i, i, i, d, d] + [vp] * 14
    lib.swe_ens_set_precision.argtypes = [i]
    for name in ("swe_ens_set_state", "swe_ens_get_state", "swe_ens_tune", "swe_ens_config",
                 "swe_ens_invariants", "swe_ens_last_timings"):
        getattr(lib, name).argtypes = [vp]
    lib.swe_ens_eval_rhs.argtypes = [vp, vp]
    lib.swe_ens_step.argtypes = [i]
    lib.swe_ens_stage.argtypes = [i]
    lib.swe_ens_set_timing.argtypes = [i]
    lib.swe_ens_use_variant.argtypes = [i, i]
    lib.swe_ens_stream.restype = vp
    lib.swe_srv_start.argtypes = [d, i]
    lib.swe_srv_add_grid.argtypes = [i, i, d, d] + [vp] * 14
    lib.swe_srv_submit.argtypes = [i, i, i, vp]
    lib.swe_srv_poll.argtypes = [i, vp]
    lib.swe_srv_fetch.argtypes = [i, vp]
    lib.swe_cuda_halo_setup.argtypes = [vp, i, vp, i]
    lib.swe_cuda_halo_pack.argtypes = [i, vp]
    lib.swe_cuda_halo_unpack.argtypes = [i, vp]
    lib.swe_srv_set_dep_limit.argtypes = [d]
    lib.swe_srv_test_withhold.argtypes = [i, i]
    lib.swe_srv_cancel.argtypes = [i]
    lib.swe_srv_stats.argtypes = [vp]
    _lib = lib
    return lib


def check(fn: str, status: int) -> None:
    if status != 0:
        raise SweError(fn, status, load().swe_cuda_last_error().decode(errors="replace"))


def kernel_launches() -> int:
    return int(load().swe_b200_kernel_launches())


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


class PSMD(ctypes.Structure):
    """Mirror of the reference's PSMD_struct (swe_config.h:187-233) with pointers
    left untyped; gh0 and dt are fType, so two variants exist."""

    _common_head = [(n, ctypes.c_int) for n in (
        "lnbr_rank", "rnbr_rank", "patch_size", "compute_size", "lhalo_size", "rhalo_size",
        "halo_pid_s", "compute_pid_s", "compute_pid_e", "halo_pid_e", "lnbr_halo_size",
        "rnbr_halo_size", "lnbr_halo_pid_e", "rnbr_halo_pid_s")] + \
        [(n, ctypes.c_void_p) for n in ("x", "y", "z", "f")]
    _common_tail = [(n, ctypes.c_void_p) for n in ("ghm", "gradghm", "p_u", "p_v", "p_w")] + \
        [("Nnbr", ctypes.c_int), ("padded_Nnbr", ctypes.c_int)] + \
        [(n, ctypes.c_void_p) for n in ("idx", "Dx", "Dy", "Dz", "L")]


class PSMD64(ctypes.Structure):
    _fields_ = PSMD._common_head + [("gh0", ctypes.c_double), ("dt", ctypes.c_double)] + PSMD._common_tail


class PSMD32(ctypes.Structure):
    _fields_ = PSMD._common_head + [("gh0", ctypes.c_float), ("dt", ctypes.c_float)] + PSMD._common_tail


class Plain:
    """The plain drop-in form (swe_cuda_*), one process-wide instance."""

    def __init__(self):
        self.lib = load()
        self.fsize = None
        self._keep = None

    # -- init ------------------------------------------------------------------------
    def init(self, fsize: int, layout: int, simd_length: int, compute_size: int, patch_size: int,
             compute_pid_s: int, nnbr: int, padded_nnbr: int, gh0: float, dt: float, arrays: dict) -> None:
        names = ("x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm", "idx", "Dx", "Dy", "Dz", "L")
        ptrs = []
        for n in names:
            a = arrays[n]
            ptrs.append(a if isinstance(a, int) else _p(a))
        check("swe_cuda_init", self.lib.swe_cuda_init(
            fsize, layout, simd_length, compute_size, patch_size, compute_pid_s, nnbr, padded_nnbr,
            float(gh0), float(dt), *ptrs))
        self.fsize, self.layout, self.S = fsize, layout, simd_length
        self.compute_size, self.patch_size = compute_size, patch_size
        self.dtype = np.float64 if fsize == 8 else np.float32

    def init_model(self, model, prec: str = "fp64") -> None:
        """Canonical CFDL layout from a swe_input.SweModel (node-major, idx 0-based)."""
        dt = np.float64 if prec == "fp64" else np.float32
        arrs = {k: np.ascontiguousarray(getattr(model, k), dtype=dt) for k in
                ("x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm", "Dx", "Dy", "Dz", "L")}
        arrs["idx"] = np.ascontiguousarray(model.idx, dtype=np.int32)
        self._keep = arrs
        fs = np.dtype(dt).itemsize
        self.init(fs, SWE_LAYOUT_CFDL, 1, model.N, model.N, 0, model.Nnbr, model.Nnbr,
                  float(model.gh0), float(model.dt), arrs)

    def init_psmd(self, psmd_addr: int, fsize: int, layout: int, simd_length: int) -> None:
        """Forward a reference PSMD_struct (what swe_cuda_init_psmd does in C)."""
        p = (PSMD64 if fsize == 8 else PSMD32).from_address(psmd_addr)
        arrays = {n: getattr(p, n) for n in
                  ("x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm", "idx", "Dx", "Dy", "Dz", "L")}
        self.init(fsize, layout, simd_length, p.compute_size, p.patch_size, p.compute_pid_s,
                  p.Nnbr, p.padded_Nnbr, float(p.gh0), float(p.dt), arrays)

    # -- state / stepping ---------------------------------------------------------------
    def set_state(self, H: np.ndarray) -> None:
        H = np.ascontiguousarray(H, dtype=self.dtype)
        assert H.size == 4 * self.patch_size
        check("swe_cuda_set_state", self.lib.swe_cuda_set_state(_p(H)))
        self.lib.swe_cuda_sync()

    def set_state_ptr(self, addr: int) -> None:
        check("swe_cuda_set_state", self.lib.swe_cuda_set_state(addr))

    def get_state(self) -> np.ndarray:
        H = np.empty(4 * self.patch_size, dtype=self.dtype)
        check("swe_cuda_get_state", self.lib.swe_cuda_get_state(_p(H)))
        return H

    def get_state_ptr(self, addr: int) -> None:
        check("swe_cuda_get_state", self.lib.swe_cuda_get_state(addr))

    def eval_rhs(self, K: np.ndarray) -> np.ndarray:
        K = np.ascontiguousarray(K, dtype=self.dtype)
        assert K.size == 4 * self.patch_size
        F = np.empty(4 * self.compute_size, dtype=self.dtype)
        check("swe_cuda_eval_rhs", self.lib.swe_cuda_eval_rhs(_p(K), _p(F)))
        return F

    def rk_substep(self, substep_id: int) -> None:
        check("swe_cuda_rk_substep", self.lib.swe_cuda_rk_substep(int(substep_id)))

    def step(self, nsteps: int) -> None:
        check("swe_cuda_step", self.lib.swe_cuda_step(int(nsteps)))

    def sync(self) -> None:
        check("swe_cuda_sync", self.lib.swe_cuda_sync())

    def set_timing(self, on: bool) -> None:
        check("swe_cuda_set_timing", self.lib.swe_cuda_set_timing(1 if on else 0))

    def timings(self) -> tuple[float, int, float]:
        out = np.zeros(3)
        check("swe_cuda_last_timings", self.lib.swe_cuda_last_timings(_p(out)))
        return float(out[0]), int(out[1]), float(out[2])

    def stream(self) -> int:
        return int(self.lib.swe_cuda_stream() or 0)

    def halo_setup(self, send_rows: np.ndarray, recv_rows: np.ndarray) -> None:
        """Patch rows this rank sends (its compute rows other ranks read) and receives."""
        s = np.ascontiguousarray(send_rows, dtype=np.int32)
        r = np.ascontiguousarray(recv_rows, dtype=np.int32)
        check("swe_cuda_halo_setup", self.lib.swe_cuda_halo_setup(_p(s), len(s), _p(r), len(r)))

    def halo_pack(self, substep_id: int, send_ptr: int) -> None:
        """Send rows of the buffer substep `substep_id` reads -> a [n_send][4] device buffer."""
        check("swe_cuda_halo_pack", self.lib.swe_cuda_halo_pack(int(substep_id), send_ptr))

    def halo_unpack(self, substep_id: int, recv_ptr: int) -> None:
        """A [n_recv][4] device buffer -> the receive rows of that buffer."""
        check("swe_cuda_halo_unpack", self.lib.swe_cuda_halo_unpack(int(substep_id), recv_ptr))

    def select_kernel(self, which: int) -> None:
        """0: bulk-copy pipelined stage kernel, 1: register-streaming kernel, 2 / 3 / 4: pipelined with
        64- / 32- / 16-node tiles, 5: node-per-lane kernel, 6 + s: node-per-lane shape s (lane_shape())."""
        check("swe_cuda_select_kernel", self.lib.swe_cuda_select_kernel(int(which)))

    @staticmethod
    def lane_shape(lanes_per_node: int, ctas_per_sm: int = 4, l2_prefetch: bool = False) -> int:
        """select_kernel code of a node-per-lane shape (3, 4 or 5 CTAs per SM)."""
        li = {1: 0, 2: 1, 4: 2}[lanes_per_node]
        if ctas_per_sm == 3:
            return 18 + li + (3 if l2_prefetch else 0)
        s = li + (3 if ctas_per_sm == 5 else 0) + (6 if l2_prefetch else 0)
        return 6 + s

    def set_index_width(self, bits: int) -> None:
        """16: the node-per-lane kernel reads stencil rows as 16-bit offsets from each node's
        own row (the default when every offset fits); 32: as the 32-bit indices."""
        check("swe_cuda_set_index_width", self.lib.swe_cuda_set_index_width(int(bits)))

    def kernel_info(self) -> dict:
        out = np.zeros(9, dtype=np.int32)
        check("swe_cuda_kernel_info", self.lib.swe_cuda_kernel_info(_p(out)))
        return {"in_use": ("pipelined", "register", "lane")[int(out[0])], "pipelined_available": bool(out[1]),
                "pipelined_tile": int(out[1]), "lanes_per_node": int(out[4]), "l2_prefetch": bool(out[6]),
                "ctas_per_sm": int(out[7]), "index_offsets_16bit": bool(out[8]),
                "tune_us": {"pipelined": out[2] / 1e3, "register": out[3] / 1e3, "lane": out[5] / 1e3}}

    def invariants(self) -> np.ndarray:
        """FP64 (mass, energy); raises SweError (SWE_ERR_NONFINITE) when the state holds NaN/Inf."""
        out = np.zeros(2)
        check("swe_cuda_invariants", self.lib.swe_cuda_invariants(_p(out)))
        return out

    def hist_open(self, path: str, interval: int) -> None:
        """Append the state to `path` every `interval` RK4 steps (see swe_b200.history)."""
        check("swe_hist_open", self.lib.swe_hist_open(os.fsencode(path), int(interval)))

    def hist_close(self) -> None:
        check("swe_hist_close", self.lib.swe_hist_close())

    def hist_stats(self) -> dict:
        out = np.zeros(4, dtype=np.int64)
        check("swe_hist_stats", self.lib.swe_hist_stats(_p(out)))
        return {"open": bool(out[0]), "records": int(out[1]), "bytes": int(out[2]), "steps": int(out[3])}

    def finalize(self) -> None:
        check("swe_cuda_finalize", self.lib.swe_cuda_finalize())


class Ensemble:
    """The batched-ensemble form (swe_ens_*): `members` states on one grid."""

    def __init__(self):
        self.lib = load()
        self._keep = None

    def init(self, model, members: int) -> None:
        arrs = {k: np.ascontiguousarray(getattr(model, k), dtype=np.float64) for k in
                ("Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm")}
        idx = np.ascontiguousarray(model.idx, dtype=np.int32)
        self._keep = (arrs, idx)
        check("swe_ens_init", self.lib.swe_ens_init(
            members, model.N, model.Nnbr, float(model.gh0), float(model.dt), _p(idx),
            *[_p(arrs[k]) for k in ("Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm",
                                    "p_u", "p_v", "p_w", "gradghm")]))
        self.members, self.n = members, model.N

    def set_state(self, H: np.ndarray) -> None:
        H = np.ascontiguousarray(H, dtype=np.float64).reshape(self.members, self.n, 4)
        check("swe_ens_set_state", self.lib.swe_ens_set_state(_p(H)))
        self.sync()

    def get_state(self) -> np.ndarray:
        H = np.empty((self.members, self.n, 4))
        check("swe_ens_get_state", self.lib.swe_ens_get_state(_p(H)))
        return H

    def set_state_ptr(self, addr: int) -> None:
        """[members][n][4] FP64 from a host address (pinned for full PCIe speed); asynchronous."""
        check("swe_ens_set_state", self.lib.swe_ens_set_state(addr))

    def get_state_ptr(self, addr: int) -> None:
        """[members][n][4] FP64 to a host address; synchronises."""
        check("swe_ens_get_state", self.lib.swe_ens_get_state(addr))

    def eval_rhs(self, K: np.ndarray) -> np.ndarray:
        K = np.ascontiguousarray(K, dtype=np.float64).reshape(self.members, self.n, 4)
        F = np.empty_like(K)
        check("swe_ens_eval_rhs", self.lib.swe_ens_eval_rhs(_p(K), _p(F)))
        return F

    def step(self, nsteps: int) -> None:
        check("swe_ens_step", self.lib.swe_ens_step(int(nsteps)))

    def stage(self, s: int) -> None:
        check("swe_ens_stage", self.lib.swe_ens_stage(int(s)))

    def sync(self) -> None:
        check("swe_ens_sync", self.lib.swe_ens_sync())

    # order of swe_ens_tune's table: (tile nodes, members per CTA)
    TUNE_VARIANTS = ((32, 64), (32, 32), (16, 64), (16, 32))

    def tune(self) -> np.ndarray:
        """ms per RK4 step of each variant in TUNE_VARIANTS order (-1: not usable)."""
        ms = np.zeros(4)
        check("swe_ens_tune", self.lib.swe_ens_tune(_p(ms)))
        return ms

    def use_variant(self, tile_nodes: int, members_per_cta: int) -> None:
        check("swe_ens_use_variant", self.lib.swe_ens_use_variant(tile_nodes, members_per_cta))

    PRECISIONS = ("tf32x3", "bf16x3", "fp16x3")

    def set_precision(self, name: str) -> None:
        """Stencil products in 3xTF32 ("tf32x3", the default), split BF16 ("bf16x3") or split
        FP16 with power-of-two scales ("fp16x3")."""
        if name not in self.PRECISIONS:
            raise ValueError(f"precision must be one of {self.PRECISIONS}, got {name!r}")
        check("swe_ens_set_precision", self.lib.swe_ens_set_precision(self.PRECISIONS.index(name)))

    def config(self) -> dict:
        out = np.zeros(6, dtype=np.int32)
        check("swe_ens_config", self.lib.swe_ens_config(_p(out)))
        return {"tile_nodes": int(out[0]), "members_per_cta": int(out[1]),
                "max_rows_per_tile": int(out[2]), "tiles": int(out[3]),
                "precision": self.PRECISIONS[int(out[4])], "chunks": int(out[5])}

    def invariants(self) -> np.ndarray:
        """FP64 (mass, energy) per member; raises SweError (SWE_ERR_NONFINITE) naming the first
        member whose state holds NaN/Inf."""
        out = np.zeros((self.members, 2))
        check("swe_ens_invariants", self.lib.swe_ens_invariants(_p(out)))
        return out

    def set_timing(self, on: bool) -> None:
        check("swe_ens_set_timing", self.lib.swe_ens_set_timing(1 if on else 0))

    def last_step_seconds(self) -> float:
        out = np.zeros(1)
        check("swe_ens_last_timings", self.lib.swe_ens_last_timings(_p(out)))
        return float(out[0])

    def stream(self) -> int:
        return int(self.lib.swe_ens_stream() or 0)

    def finalize(self) -> None:
        check("swe_ens_finalize", self.lib.swe_ens_finalize())


class Server:
    """The serving form (swe_srv_*): continuous batching of forecast requests."""

    STAT_NAMES = ("kernel_launches", "admitted", "completed", "bytes_in_use", "peak_bytes", "budget",
                  "items_done", "queued", "running", "dependency_failures")

    def __init__(self, budget_bytes: float, max_requests: int = 256):
        self.lib = load()
        check("swe_srv_start", self.lib.swe_srv_start(float(budget_bytes), int(max_requests)))
        self.grids = {}
        self.meta = {}
        self._keep = []

    def add_grid(self, model) -> int:
        arrs = {k: np.ascontiguousarray(getattr(model, k), dtype=np.float64) for k in
                ("Dx", "Dy", "Dz", "L", "x", "y", "z", "f", "ghm", "p_u", "p_v", "p_w", "gradghm")}
        idx = np.ascontiguousarray(model.idx, dtype=np.int32)
        gid = self.lib.swe_srv_add_grid(model.N, model.Nnbr, float(model.gh0), float(model.dt), _p(idx),
                                        *[_p(arrs[k]) for k in ("Dx", "Dy", "Dz", "L", "x", "y", "z", "f",
                                                                "ghm", "p_u", "p_v", "p_w", "gradghm")])
        if gid < 0:
            check("swe_srv_add_grid", -gid)
        self.grids[gid] = model.N
        return gid

    def submit(self, grid: int, H0: np.ndarray, nsteps: int) -> int:
        H0 = np.ascontiguousarray(H0, dtype=np.float64).reshape(-1, self.grids[grid], 4)
        rid = self.lib.swe_srv_submit(grid, H0.shape[0], int(nsteps), _p(H0))
        if rid < 0:
            check("swe_srv_submit", -rid)
        self.meta[rid] = (grid, H0.shape[0])
        return rid

    def poll(self, rid: int):
        """(state, admit_s, done_s): state 0 queued/running, 1 done, 2 cancelled."""
        t = np.zeros(2)
        st = self.lib.swe_srv_poll(rid, _p(t))
        if st < 0:
            check("swe_srv_poll", -st)
        return st, float(t[0]), float(t[1])

    def fetch(self, rid: int) -> np.ndarray:
        grid, members = self.meta.pop(rid)
        H = np.empty((members, self.grids[grid], 4))
        check("swe_srv_fetch", self.lib.swe_srv_fetch(rid, _p(H)))
        return H

    def cancel(self, rid: int) -> None:
        check("swe_srv_cancel", self.lib.swe_srv_cancel(rid))

    def set_dep_limit(self, seconds: float) -> None:
        """Limit of a work item's wait for its request's previous stage."""
        check("swe_srv_set_dep_limit", self.lib.swe_srv_set_dep_limit(ctypes.c_double(seconds)))

    def test_withhold(self, rid: int, stage_index: int) -> None:
        """Test hook: the first work item of stage `stage_index` (step * 4 + stage) of
        request `rid` (of the next request submitted, when rid < 0) is never queued, so
        the following stage's wait runs out."""
        check("swe_srv_test_withhold", self.lib.swe_srv_test_withhold(int(rid), int(stage_index)))

    def stats(self) -> dict:
        out = np.zeros(10)
        check("swe_srv_stats", self.lib.swe_srv_stats(_p(out)))
        return dict(zip(self.STAT_NAMES, out.tolist()))

    def wait(self, rids, timeout: float = 120.0) -> dict:
        """Poll until every request in rids is done or cancelled; {rid: (state, admit_s, done_s)}."""
        import time as _t

        t0 = _t.time()
        res = {}
        while len(res) < len(rids):
            for r in rids:
                if r not in res:
                    st = self.poll(r)
                    if st[0] != 0:
                        res[r] = st
            if _t.time() - t0 > timeout:
                raise TimeoutError(f"requests not done after {timeout}s: {sorted(set(rids) - set(res))}")
            _t.sleep(0.0005)
        return res

    def stop(self) -> None:
        check("swe_srv_stop", self.lib.swe_srv_stop())
