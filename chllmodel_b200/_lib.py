"""ctypes binding of libchll_mod.so (declared in include/chll_mod.h).

The library is the only compute path: there is no CPU fallback.  Loading
fails loudly if the shared library has not been built, and every extension
call raises ``ChllError`` with the library's own message when it fails
(including "no CUDA device available" on a machine without a GPU).
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libchll_mod.so")

CHLL_OK, CHLL_EINVAL, CHLL_ECUDA, CHLL_ENOMEM, CHLL_EDEVICE, CHLL_ERANGE = range(6)
CHLL_OPEN, CHLL_PERIODIC = 0, 1
ROW_LEN = 16
ROW_ETOT, ROW_ETA, ROW_PACCEPT, ROW_FACCEPT, ROW_D = 0, 1, 2, 3, 4
ROW_ENERGY, ROW_SUM_S, ROW_QXX, ROW_ETOT_SUM, ROW_STEP, ROW_NSITES = 5, 6, 7, 13, 14, 15

# Every symbol include/chll_mod.h declares.
EXPORTS = (
    "init", "run", "chll_last_status", "chll_last_error", "chll_set_seed", "chll_version",
    "chll_run_ex", "chll_lattice_create", "chll_lattice_destroy", "chll_lattice_set_stream",
    "chll_lattice_sync", "chll_lattice_init_random", "chll_lattice_upload_f64",
    "chll_lattice_download_f64", "chll_lattice_upload_f4", "chll_lattice_download_f4",
    "chll_lattice_storage", "chll_lattice_set_control", "chll_lattice_get_control",
    "chll_lattice_sweep", "chll_lattice_pass", "chll_lattice_observe",
    "chll_lattice_energy_grad", "chll_lattice_reserve_rows", "chll_lattice_measure",
    "chll_lattice_read_rows", "chll_energy_grad_noalloc", "chll_lattice_quench",
    "chll_lattice_set_kernel", "chll_lattice_shell_corr", "chll_lattice_projection",
    "chll_lattice_create_slab", "chll_lattice_slab_plane", "chll_lattice_counters",
    "chll_lattice_control_update", "chll_lattice_slab_set_peers", "chll_lattice_slab_push",
    "chll_lattice_ipc_handle", "chll_ipc_open", "chll_ipc_close",
    "chll_batch_create", "chll_batch_destroy", "chll_batch_set_stream", "chll_batch_sync",
    "chll_batch_init_random", "chll_batch_upload_f4", "chll_batch_download_f4", "chll_batch_run",
    "chll_batch_moments", "chll_batch_info", "chll_batch_set_tuning", "chll_batch_autotune",
    "chll_batch_set_wave_bytes", "chll_batch_get_tuning", "chll_batch_set_wait_limit",
    "chll_batch_set_pairing", "chll_batch_get_pairing", "chll_batch_set_pooled",
    "chll_batch_get_pooled",
)


def torch_stream_handle(stream=None) -> int:
    """The CUDA stream handle of a torch stream (default: the current one) for
    the set_stream calls: torch's default stream is handle 0, which the
    library reads as "the lattice's own stream", so it becomes
    cudaStreamLegacy (1), the same default stream by its explicit name."""
    import torch

    h = (stream if stream is not None else torch.cuda.current_stream()).cuda_stream
    return h if h else 1


class ChllError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"libchll_mod error {code}: {message}")
        self.code = code


class RunConfig(ct.Structure):
    """chll_run_config."""

    _fields_ = [
        ("kT", ct.c_double), ("K", ct.c_double), ("g", ct.c_double), ("eps", ct.c_double),
        ("d", ct.c_double), ("seed", ct.c_uint64), ("replica", ct.c_uint32),
        ("boundary", ct.c_int32), ("adapt_until", ct.c_int64), ("verbose", ct.c_int32),
        ("reserved", ct.c_int32),
    ]


class Coupling(ct.Structure):
    """chll_coupling."""

    _fields_ = [("kT", ct.c_double), ("K", ct.c_double), ("g", ct.c_double),
                ("eps", ct.c_double)]


class ReplicaSpec(ct.Structure):
    """chll_replica_spec."""

    _fields_ = [
        ("ni", ct.c_int32), ("nj", ct.c_int32), ("nk", ct.c_int32), ("boundary", ct.c_int32),
        ("kT", ct.c_double), ("K", ct.c_double), ("g", ct.c_double), ("eps", ct.c_double),
        ("d", ct.c_double), ("seed", ct.c_uint64), ("replica", ct.c_uint32),
        ("reserved", ct.c_uint32),
    ]


_lib = None


def load() -> ct.CDLL:
    """Loads libchll_mod.so (building it first if nvcc is available)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        try:
            from . import build as _build

            _build.build()
        except Exception as exc:  # noqa: BLE001 - surfaced below
            raise ImportError(
                f"libchll_mod.so is not built ({LIB_PATH}) and building it failed: {exc}"
            ) from exc
    L = ct.CDLL(LIB_PATH)
    _declare(L)
    _lib = L
    return L


def _declare(L: ct.CDLL) -> None:
    P = ct.POINTER
    i32, i64, u32, u64, dbl, vp = ct.c_int, ct.c_int64, ct.c_uint32, ct.c_uint64, ct.c_double, ct.c_void_p
    f_arr = np.ctypeslib.ndpointer(dtype=np.float64, ndim=3, flags="F_CONTIGUOUS")
    i_arr = np.ctypeslib.ndpointer(dtype=np.int32, ndim=3, flags="F_CONTIGUOUS")
    i1 = np.ctypeslib.ndpointer(dtype=np.int32, ndim=1, flags="F_CONTIGUOUS")
    f2 = np.ctypeslib.ndpointer(dtype=np.float64, ndim=2, flags="F_CONTIGUOUS")
    # reference entry points, with the argtypes of chll/chll.py:9-36
    L.init.argtypes = [f_arr, f_arr, f_arr, i_arr, i_arr, i1, i1, P(i32), P(i32), P(i32), P(i32)]
    L.init.restype = None
    L.run.argtypes = [P(i32), P(i32), P(i32), f_arr, f_arr, f_arr, i_arr, i_arr, i1, i1,
                      P(dbl), P(dbl), P(dbl), P(dbl), P(i32), P(i32), P(i32), P(i32), i1, f2]
    L.run.restype = None
    L.chll_last_status.argtypes = []
    L.chll_last_status.restype = i32
    L.chll_last_error.argtypes = []
    L.chll_last_error.restype = ct.c_char_p
    L.chll_set_seed.argtypes = [u64]
    L.chll_set_seed.restype = None
    L.chll_version.argtypes = []
    L.chll_version.restype = ct.c_char_p
    L.chll_run_ex.argtypes = [P(RunConfig), i32, i32, i32, vp, vp, vp, vp, i32, i32, i32, vp, vp,
                              vp, P(dbl)]
    L.chll_run_ex.restype = i32
    L.chll_lattice_create.argtypes = [i32, i32, i32, i32, P(vp)]
    L.chll_lattice_create.restype = i32
    L.chll_lattice_destroy.argtypes = [vp]
    L.chll_lattice_destroy.restype = None
    L.chll_lattice_set_stream.argtypes = [vp, vp]
    L.chll_lattice_sync.argtypes = [vp]
    L.chll_lattice_init_random.argtypes = [vp, u64, u32]
    L.chll_lattice_upload_f64.argtypes = [vp, vp, vp, vp, vp]
    L.chll_lattice_download_f64.argtypes = [vp, vp, vp, vp, vp]
    L.chll_lattice_upload_f4.argtypes = [vp, vp]
    L.chll_lattice_download_f4.argtypes = [vp, vp]
    L.chll_lattice_storage.argtypes = [vp, P(vp), P(vp), P(i64), P(ct.c_int32)]
    L.chll_lattice_set_control.argtypes = [vp, dbl, i64, i64]
    L.chll_lattice_get_control.argtypes = [vp, P(dbl), P(i64), P(dbl), P(dbl)]
    L.chll_lattice_sweep.argtypes = [vp, P(Coupling), u64, u32, i32]
    L.chll_lattice_pass.argtypes = [vp, P(Coupling), u64, u32, i32]
    L.chll_lattice_observe.argtypes = [vp, P(Coupling), vp]
    L.chll_lattice_energy_grad.argtypes = [vp, P(Coupling), vp, i32, vp]
    L.chll_lattice_set_kernel.argtypes = [vp, i32]
    L.chll_lattice_set_kernel.restype = i32
    L.chll_lattice_quench.argtypes = [vp, P(Coupling), dbl, i32]
    L.chll_lattice_quench.restype = i32
    L.chll_lattice_create_slab.argtypes = [i32, i32, i32, i32, i32, i32, P(vp)]
    L.chll_lattice_slab_plane.argtypes = [vp, i32, i32, P(vp), P(i64)]
    L.chll_lattice_counters.argtypes = [vp, P(vp)]
    L.chll_lattice_control_update.argtypes = [vp, i32]
    L.chll_lattice_slab_set_peers.argtypes = [vp, vp, vp, vp, vp]
    L.chll_lattice_slab_push.argtypes = [vp, i32]
    L.chll_lattice_ipc_handle.argtypes = [vp, vp, P(u64)]
    L.chll_ipc_open.argtypes = [vp, P(vp)]
    L.chll_ipc_close.argtypes = [vp]
    for name in ("chll_lattice_create_slab", "chll_lattice_slab_plane", "chll_lattice_counters",
                 "chll_lattice_control_update", "chll_lattice_slab_set_peers",
                 "chll_lattice_slab_push", "chll_lattice_ipc_handle", "chll_ipc_open",
                 "chll_ipc_close"):
        getattr(L, name).restype = i32
    L.chll_lattice_shell_corr.argtypes = [vp, i32, i32, vp, vp, vp]
    L.chll_lattice_shell_corr.restype = i32
    L.chll_lattice_projection.argtypes = [vp, vp, vp, P(ct.c_longlong), P(i32)]
    L.chll_lattice_projection.restype = i32
    L.chll_lattice_reserve_rows.argtypes = [vp, i32]
    L.chll_lattice_measure.argtypes = [vp, P(Coupling), i32]
    L.chll_lattice_read_rows.argtypes = [vp, vp, i32, i32]
    for name in ("chll_lattice_set_stream", "chll_lattice_sync", "chll_lattice_init_random",
                 "chll_lattice_upload_f64", "chll_lattice_download_f64", "chll_lattice_upload_f4",
                 "chll_lattice_download_f4", "chll_lattice_storage", "chll_lattice_set_control",
                 "chll_lattice_get_control", "chll_lattice_sweep", "chll_lattice_pass",
                 "chll_lattice_observe", "chll_lattice_energy_grad", "chll_lattice_reserve_rows",
                 "chll_lattice_measure", "chll_lattice_read_rows"):
        getattr(L, name).restype = i32
    L.chll_energy_grad_noalloc.argtypes = [vp, vp, i32, i32, i32, i32, P(Coupling), i32, vp, vp,
                                           vp]
    L.chll_energy_grad_noalloc.restype = i32
    L.chll_batch_create.argtypes = [P(ReplicaSpec), i32, P(vp)]
    L.chll_batch_create.restype = i32
    L.chll_batch_destroy.argtypes = [vp]
    L.chll_batch_destroy.restype = None
    L.chll_batch_set_stream.argtypes = [vp, vp]
    L.chll_batch_sync.argtypes = [vp]
    L.chll_batch_init_random.argtypes = [vp]
    L.chll_batch_run.argtypes = [vp, i32, i32, i32]
    L.chll_batch_moments.argtypes = [vp, vp]
    L.chll_batch_download_f4.argtypes = [vp, i32, vp]
    L.chll_batch_upload_f4.argtypes = [vp, i32, vp]
    L.chll_batch_info.argtypes = [vp, P(i64), P(ct.c_int32), P(ct.c_int32), P(ct.c_int32)]
    L.chll_batch_set_tuning.argtypes = [vp, i32, i32]
    L.chll_batch_autotune.argtypes = [vp, i32, P(i32), P(i32), P(dbl)]
    L.chll_batch_set_wave_bytes.argtypes = [vp, i64]
    L.chll_batch_set_wait_limit.argtypes = [vp, ct.c_uint64]
    L.chll_batch_set_pairing.argtypes = [vp, i32]
    L.chll_batch_get_pairing.argtypes = [vp, P(i32)]
    L.chll_batch_set_pooled.argtypes = [vp, i32]
    L.chll_batch_get_pooled.argtypes = [vp, P(i32)]
    L.chll_batch_get_tuning.argtypes = [vp, P(ct.c_int32), P(ct.c_int32), P(i64), P(ct.c_int32)]
    for name in ("chll_batch_set_stream", "chll_batch_sync", "chll_batch_init_random",
                 "chll_batch_run", "chll_batch_moments", "chll_batch_download_f4",
                 "chll_batch_upload_f4", "chll_batch_info", "chll_batch_set_tuning",
                 "chll_batch_autotune", "chll_batch_set_wave_bytes", "chll_batch_get_tuning",
                 "chll_batch_set_wait_limit", "chll_batch_set_pairing", "chll_batch_get_pairing",
                 "chll_batch_set_pooled", "chll_batch_get_pooled"):
        getattr(L, name).restype = i32


def check(rc: int) -> None:
    if rc != CHLL_OK:
        msg = load().chll_last_error().decode(errors="replace")
        raise ChllError(rc, msg)


def last_error() -> str:
    return load().chll_last_error().decode(errors="replace")
