"""icempm_b200 -- B200-native 2D MLS-MPM substep for iceMPM.

Python host mirror of the reference's device-layer API over the C ABI of
``include/icempm.h`` (``libicempm.so``, built in-tree for sm_100a):

* :class:`SimParams` -- ``icy::SimParams`` (simulation/parameters_sim.h:19-90),
  byte-identical 432-byte layout, with ``Reset``/``ParseFile`` and the derived
  constants of simulation/parameters_sim.cpp.
* :class:`GPU_Implementation5` -- the member functions and public data members
  of simulation/gpu_implementation5.h:40-72. Like the reference, every failure
  raises ``RuntimeError``.
* :class:`Model` -- ``icy::Model`` (simulation/model.h:26-52): ``Step`` runs one
  frame of ``UpdateEveryNthStep`` substeps (simulation/model.cpp:11-47).

The library is required: importing works without it, but every call that
needs it raises ``RuntimeError`` naming the missing file. There is no CPU
fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from typing import Callable, Optional

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libicempm.so")

# forms of icm_run_substeps
FORM_FP64_STEPWISE = 0
FORM_FP64 = 1
FORM_FP32 = 2
FORM_FP32_SURROGATE = 3
FORM_FP32_COMPENSATED = 4
FORM_NAMES = {FORM_FP64_STEPWISE: "fp64-stepwise", FORM_FP64: "fp64", FORM_FP32: "fp32",
              FORM_FP32_SURROGATE: "fp32-surrogate", FORM_FP32_COMPENSATED: "fp32-compensated"}

# tile variants of the fused forms (nodes)
TILE_VARIANTS = {0: (16, 8), 1: (16, 16), 2: (32, 8), 3: (32, 16)}

# particle SoA rows (parameters_sim.h:27-35)
IDX_UTILITY, IDX_P, IDX_Q, IDX_JP_INV, IDX_POSX, IDX_VELX, IDX_FE00, IDX_BP00 = 0, 1, 2, 3, 4, 6, 8, 12
N_PTS_ARRAYS, N_GRID_ARRAYS = 16, 3


class SimParams(C.Structure):
    """``icy::SimParams`` with the reference's field order and padding."""

    _fields_ = [
        ("grid_array", C.c_void_p), ("indenter_force_accumulator", C.c_void_p), ("pts_array", C.c_void_p),
        ("nPtsPitch", C.c_size_t), ("nGridPitch", C.c_size_t),
        ("n_indenter_subdivisions", C.c_int), ("tpb_P2G", C.c_int), ("tpb_Upd", C.c_int), ("tpb_G2P", C.c_int),
        ("nPts", C.c_int), ("GridX", C.c_int), ("GridY", C.c_int), ("GridTotal", C.c_int),
        ("GridXDimension", C.c_double),
        ("InitialTimeStep", C.c_double), ("SimulationEndTime", C.c_double),
        ("Gravity", C.c_double), ("Density", C.c_double), ("PoissonsRatio", C.c_double), ("YoungsModulus", C.c_double),
        ("lambda_", C.c_double), ("mu", C.c_double), ("kappa", C.c_double),
        ("IceCompressiveStrength", C.c_double), ("IceTensileStrength", C.c_double), ("IceShearStrength", C.c_double),
        ("NACC_beta", C.c_double), ("NACC_M", C.c_double), ("NACC_Msq", C.c_double),
        ("DP_tan_phi", C.c_double), ("DP_threshold_p", C.c_double),
        ("cellsize", C.c_double), ("cellsize_inv", C.c_double), ("Dp_inv", C.c_double),
        ("UpdateEveryNthStep", C.c_int),
        ("IndDiameter", C.c_double), ("IndRSq", C.c_double), ("IndVelocity", C.c_double), ("IndDepth", C.c_double),
        ("xmin", C.c_double), ("xmax", C.c_double), ("ymin", C.c_double), ("ymax", C.c_double),
        ("nxmin", C.c_int), ("nxmax", C.c_int), ("nymin", C.c_int), ("nymax", C.c_int),
        ("ParticleVolume", C.c_double), ("ParticleMass", C.c_double), ("ParticleViewSize", C.c_double),
        ("SimulationStep", C.c_int),
        ("SimulationTime", C.c_double),
        ("indenter_x", C.c_double), ("indenter_x_initial", C.c_double),
        ("indenter_y", C.c_double), ("indenter_y_initial", C.c_double),
        ("Volume", C.c_double),
        ("SetupType", C.c_int),
        ("GrainVariability", C.c_double),
        ("UseWarpLevelReduction", C.c_int), ("SortPointsByGridCell", C.c_int),
    ]

    pi = 3.14159265358979323846
    dim = 2
    nGridArrays = N_GRID_ARRAYS
    nPtsArrays = N_PTS_ARRAYS

    def Reset(self) -> None:
        _lib().icm_params_reset(C.byref(self))

    def ParseFile(self, fileName: str) -> str:
        """Parses a JSON configuration; returns its InputRawPoints entry."""
        buf = C.create_string_buffer(4096)
        _check(_lib().icm_params_parse_file(C.byref(self), fileName.encode(), buf, len(buf)))
        return buf.value.decode()

    def ParseString(self, text: str) -> str:
        buf = C.create_string_buffer(4096)
        _check(_lib().icm_params_parse_string(C.byref(self), text.encode(), buf, len(buf)))
        return buf.value.decode()

    def ComputeLame(self) -> None:
        _lib().icm_params_compute_lame(C.byref(self))

    def ComputeCamClayParams2(self) -> None:
        _lib().icm_params_compute_camclay(C.byref(self))

    def ComputeHelperVariables(self) -> None:
        _lib().icm_params_compute_helpers(C.byref(self))

    def ComputeIntegerBlockCoords(self) -> None:
        _lib().icm_params_compute_block_coords(C.byref(self))

    def PointsPerCell(self) -> float:
        return self.nPts / (self.Volume / (self.cellsize * self.cellsize))

    def AnimationFrameNumber(self) -> int:
        return self.SimulationStep // self.UpdateEveryNthStep

    def IndenterArraySize(self) -> int:
        return 8 * self.n_indenter_subdivisions * 2

    def copy(self) -> "SimParams":
        c = SimParams()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(SimParams))
        return c

    def to_bytes(self) -> bytes:
        return C.string_at(C.byref(self), C.sizeof(SimParams))

    @classmethod
    def from_bytes(cls, b: bytes) -> "SimParams":
        if len(b) != C.sizeof(cls):
            raise ValueError("SimParams size mismatch")
        c = cls()
        C.memmove(C.byref(c), b, len(b))
        return c


assert C.sizeof(SimParams) == 432, C.sizeof(SimParams)


class BlockDesc(C.Structure):
    _fields_ = [("cells_x", C.c_int), ("cells_y", C.c_int), ("ind_y_above_floor", C.c_double),
                ("grain_size", C.c_double), ("seed", C.c_uint64)]


_LIB = None
_LIB_LOCK = threading.Lock()


def _lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    with _LIB_LOCK:
        if _LIB is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m icempm_b200.build` "
                                   "(there is no CPU fallback)")
            L = C.CDLL(LIB_PATH)
            vp, i, d, sz = C.c_void_p, C.c_int, C.c_double, C.c_size_t
            P = C.POINTER(SimParams)
            sigs = {
                "icm_last_error": (C.c_char_p, []), "icm_version": (C.c_char_p, []),
                "icm_params_reset": (None, [P]),
                "icm_params_parse_file": (i, [P, C.c_char_p, C.c_char_p, sz]),
                "icm_params_parse_string": (i, [P, C.c_char_p, C.c_char_p, sz]),
                "icm_params_compute_lame": (None, [P]), "icm_params_compute_camclay": (None, [P]),
                "icm_params_compute_helpers": (None, [P]), "icm_params_compute_block_coords": (None, [P]),
                "icm_pitch_elems": (sz, [sz]),
                "icm_scene_block": (i, [P, C.POINTER(BlockDesc), vp, C.POINTER(C.c_int)]),
                "icm_create": (i, [C.POINTER(vp), i]), "icm_destroy": (i, [vp]),
                "icm_set_form": (i, [vp, i]), "icm_get_form": (i, [vp]),
                "icm_set_tile": (i, [vp, i, i]), "icm_get_tile": (i, [vp, C.POINTER(i), C.POINTER(i)]),
                "icm_allocate_arrays": (i, [vp, P, sz, sz]),
                "icm_update_constants": (i, [vp, P, i]),
                "icm_transfer_points_to_device": (i, [vp, vp]),
                "icm_reset_grid": (i, [vp]), "icm_reset_indenter_force_accumulator": (i, [vp]),
                "icm_p2g": (i, [vp]), "icm_update_nodes": (i, [vp, d, d]), "icm_g2p": (i, [vp, i]),
                "icm_transfer_from_device": (i, [vp, vp, vp, vp, vp, vp]),
                "icm_synchronize": (i, [vp]),
                "icm_transfer_grid_to_device": (i, [vp, vp]), "icm_transfer_grid_from_device": (i, [vp, vp]),
                "icm_run_substeps": (i, [vp, P, i]),
                "icm_force_history": (i, [vp, vp, i]),
                "icm_fp64_redo_count": (i, [vp, C.POINTER(C.c_ulonglong)]),
                "icm_stray_count": (i, [vp, C.POINTER(C.c_ulonglong)]),
                "icm_set_rebin_interval": (i, [vp, i]),
                "icm_set_tile_split": (i, [vp, i, d]),
                "icm_record_start": (i, [vp]), "icm_record_stop": (i, [vp]),
                "icm_elapsed_ms": (i, [vp, C.POINTER(C.c_float)]),
                "icm_stream": (vp, [vp]),
                "icm_kernel_timing": (i, [vp, i]),
                "icm_kernel_time": (i, [vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
                "icm_host_alloc": (i, [C.POINTER(vp), sz]), "icm_host_free": (i, [vp]),
                "icm_cycle_events": (i, [vp, C.POINTER(vp), C.POINTER(vp)]),
                "icm_save_snapshot": (i, [P, vp, vp, C.c_char_p, C.c_char_p, sz]),
                "icm_read_snapshot_params": (i, [C.c_char_p, P]),
                "icm_read_snapshot": (i, [C.c_char_p, vp, sz, vp, sz]),
                "icm_save_pq": (i, [P, vp, C.c_char_p, C.c_char_p, sz]),
                "icm_load_raw_points": (i, [P, C.c_char_p, vp, C.POINTER(C.c_int)]),
            }
            for name, (res, args) in sigs.items():
                f = getattr(L, name)
                f.restype = res
                f.argtypes = args
            _LIB = L
    return _LIB


def library():
    """The loaded libicempm.so (ctypes handle)."""
    return _lib()


def _check(rc: int) -> None:
    if rc != 0:
        raise RuntimeError(f"icempm error {rc}: {_lib().icm_last_error().decode()}")


def pitch_elems(n: int) -> int:
    return int(_lib().icm_pitch_elems(n))


def make_block(prms: SimParams, cells_x: int, cells_y: int, ind_y_above_floor: float = 0.2,
               grain_size: float = 0.05, seed: int = 12345, out: Optional[np.ndarray] = None) -> np.ndarray:
    """Fills prms with a seeded synthetic ice block and returns its particle
    SoA (16 x pitch doubles), standing in for SnapshotManager::LoadRawPoints."""
    desc = BlockDesc(cells_x, cells_y, ind_y_above_floor, grain_size, seed)
    n = 4 * cells_x * cells_y
    pitch = pitch_elems(n)
    if out is None:
        out = np.zeros(pitch * N_PTS_ARRAYS, dtype=np.float64)
    elif out.size < pitch * N_PTS_ARRAYS or out.dtype != np.float64 or not out.flags.c_contiguous:
        raise ValueError("out buffer too small or not contiguous float64")
    nn = C.c_int(0)
    _check(_lib().icm_scene_block(C.byref(prms), C.byref(desc), out.ctypes.data, C.byref(nn)))
    return out


class SoA:
    """Named numpy views of a particle SoA buffer (point.cpp:8-70 accessors)."""

    def __init__(self, buf: np.ndarray, pitch: int, n: int):
        self.buf, self.pitch, self.n = buf, pitch, n
        rows = buf[: pitch * N_PTS_ARRAYS].reshape(N_PTS_ARRAYS, pitch)
        self.rows = rows
        raw = buf.view(np.uint8)
        self.crushed = raw[:n]
        self.grain = raw[pitch: pitch + 2 * n].view(np.int16)
        self.P = rows[IDX_P, :n]
        self.Q = rows[IDX_Q, :n]
        self.Jp_inv = rows[IDX_JP_INV, :n]
        self.pos = rows[IDX_POSX: IDX_POSX + 2, :n]
        self.vel = rows[IDX_VELX: IDX_VELX + 2, :n]
        self.Fe = rows[IDX_FE00: IDX_FE00 + 4, :n]
        self.Bp = rows[IDX_BP00: IDX_BP00 + 4, :n]


class GPU_Implementation5:
    """Mirror of the reference device layer (gpu_implementation5.h:40-72)."""

    def __init__(self, model: Optional["Model"] = None, device: int = 0):
        self.model = model
        self.error_code = 0
        self.transfer_completion_callback: Optional[Callable[[], None]] = None
        self.tmp_transfer_buffer: Optional[np.ndarray] = None
        self.host_side_indenter_force_accumulator: Optional[np.ndarray] = None
        self._device = device
        self._ctx = C.c_void_p(None)
        self._host_ptrs = []
        self._err_box = (C.c_int * 1)()
        self._cb_keep = None
        self.initialized = False

    # gpu_implementation5.cu:452-469
    def initialize(self) -> None:
        if self.initialized:
            return
        _check(_lib().icm_create(C.byref(self._ctx), self._device))
        self.initialized = True

    def test(self) -> None:
        self.initialize()

    def synchronize(self) -> None:
        if not self.initialized:
            return
        _check(_lib().icm_synchronize(self._ctx))

    def set_form(self, form: int) -> None:
        self.initialize()
        _check(_lib().icm_set_form(self._ctx, form))

    def get_form(self) -> int:
        return int(_lib().icm_get_form(self._ctx))

    def set_tile(self, variant: int, threads: int = 128) -> None:
        self.initialize()
        _check(_lib().icm_set_tile(self._ctx, variant, threads))

    # gpu_implementation5.cu:471-479
    def cuda_update_constants(self) -> None:
        _check(_lib().icm_update_constants(self._ctx, C.byref(self.model.prms), self.error_code))

    def _alloc_pinned(self, nbytes: int) -> np.ndarray:
        nbytes = max(int(nbytes), 64)
        ptr = C.c_void_p(None)
        _check(_lib().icm_host_alloc(C.byref(ptr), nbytes))
        self._host_ptrs.append(ptr)
        arr = np.ctypeslib.as_array((C.c_double * (nbytes // 8)).from_address(ptr.value))
        return arr

    def _free_pinned(self) -> None:
        for p in self._host_ptrs:
            _lib().icm_host_free(p)
        self._host_ptrs = []
        self.tmp_transfer_buffer = None
        self.host_side_indenter_force_accumulator = None

    # gpu_implementation5.cu:481-513
    def cuda_allocate_arrays(self, nGridNodes: int, nPoints: int) -> None:
        if not self.initialized:
            self.initialize()
        self._free_pinned()
        p = self.model.prms
        _check(_lib().icm_allocate_arrays(self._ctx, C.byref(p), nGridNodes, nPoints))
        self.tmp_transfer_buffer = self._alloc_pinned(8 * p.nPtsPitch * N_PTS_ARRAYS)
        self.tmp_transfer_buffer[:] = 0
        self.host_side_indenter_force_accumulator = self._alloc_pinned(8 * 2 * 256)[: 2 * p.n_indenter_subdivisions]
        self.error_code = 0

    # gpu_implementation5.cu:515-526 (sic)
    def transfer_ponts_to_device(self) -> None:
        _check(_lib().icm_transfer_points_to_device(self._ctx, self.tmp_transfer_buffer.ctypes.data))
        self.host_side_indenter_force_accumulator[:] = 0

    def cuda_reset_grid(self) -> None:
        _check(_lib().icm_reset_grid(self._ctx))

    def cuda_reset_indenter_force_accumulator(self) -> None:
        _check(_lib().icm_reset_indenter_force_accumulator(self._ctx))

    def cuda_p2g(self) -> None:
        _check(_lib().icm_p2g(self._ctx))

    def cuda_update_nodes(self, indenter_x: float, indenter_y: float) -> None:
        _check(_lib().icm_update_nodes(self._ctx, indenter_x, indenter_y))

    def cuda_g2p(self, recordPQ: bool) -> None:
        _check(_lib().icm_g2p(self._ctx, 1 if recordPQ else 0))

    # gpu_implementation5.cu:528-552: async copies, then the completion callback
    def cuda_transfer_from_device(self) -> None:
        def _done(_user):
            self.error_code = int(self._err_box[0])
            if self.transfer_completion_callback:
                self.transfer_completion_callback()
            elif self.model is not None and self.model.processing_current_cycle_data.locked():
                # no consumer installed: the frame counts as consumed at once
                self.model.UnlockCycleMutex()

        self._cb_keep = C.CFUNCTYPE(None, C.c_void_p)(_done)
        _check(_lib().icm_transfer_from_device(
            self._ctx, self.tmp_transfer_buffer.ctypes.data,
            self.host_side_indenter_force_accumulator.ctypes.data,
            C.cast(self._err_box, C.c_void_p), C.cast(self._cb_keep, C.c_void_p), None))

    def grid_to_device(self, host_grid: np.ndarray) -> None:
        _check(_lib().icm_transfer_grid_to_device(self._ctx, np.ascontiguousarray(host_grid, np.float64).ctypes.data))

    def grid_from_device(self) -> np.ndarray:
        out = np.zeros(int(self.model.prms.nGridPitch) * N_GRID_ARRAYS, dtype=np.float64)
        _check(_lib().icm_transfer_grid_from_device(self._ctx, out.ctypes.data))
        return out

    # the substep loop of Model::Step on the device
    def run_substeps(self, prms: SimParams, n: int) -> None:
        _check(_lib().icm_run_substeps(self._ctx, C.byref(prms), n))

    def force_history(self, n: int) -> np.ndarray:
        out = np.zeros(2 * n, dtype=np.float64)
        _check(_lib().icm_force_history(self._ctx, out.ctypes.data, n))
        return out.reshape(n, 2)

    def fp64_redo_count(self) -> int:
        v = C.c_ulonglong(0)
        _check(_lib().icm_fp64_redo_count(self._ctx, C.byref(v)))
        return int(v.value)

    def set_rebin_interval(self, substeps: int) -> None:
        self.initialize()
        _check(_lib().icm_set_rebin_interval(self._ctx, substeps))

    def set_tile_split(self, max_tiles: int = 128, ratio: float = 1.3) -> None:
        """Heavy tiles run as two CTAs (icm_set_tile_split; max_tiles 0: off)."""
        self.initialize()
        _check(_lib().icm_set_tile_split(self._ctx, max_tiles, ratio))

    def stray_count(self) -> int:
        v = C.c_ulonglong(0)
        _check(_lib().icm_stray_count(self._ctx, C.byref(v)))
        return int(v.value)

    def record_start(self) -> None:
        _check(_lib().icm_record_start(self._ctx))

    def record_stop(self) -> None:
        _check(_lib().icm_record_stop(self._ctx))

    def elapsed_ms(self) -> float:
        v = C.c_float(0)
        _check(_lib().icm_elapsed_ms(self._ctx, C.byref(v)))
        return float(v.value)

    def kernel_timing(self, enable: bool) -> None:
        _check(_lib().icm_kernel_timing(self._ctx, 1 if enable else 0))

    def kernel_time(self):
        """(summed ms, launches) of the timed fused substep launches."""
        ms, n = C.c_double(0), C.c_longlong(0)
        _check(_lib().icm_kernel_time(self._ctx, C.byref(ms), C.byref(n)))
        return float(ms.value), int(n.value)

    def stream_handle(self) -> int:
        return int(_lib().icm_stream(self._ctx) or 0)

    def soa(self) -> SoA:
        p = self.model.prms
        return SoA(self.tmp_transfer_buffer, int(p.nPtsPitch), int(p.nPts))

    def close(self) -> None:
        if self.initialized:
            _lib().icm_destroy(self._ctx)
            self._ctx = C.c_void_p(None)
            self.initialized = False
        self._free_pinned()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Model:
    """Mirror of icy::Model (model.h:26-52, model.cpp:4-73)."""

    def __init__(self, device: int = 0):
        self.prms = SimParams()
        self.prms.Reset()
        self.gpu = GPU_Implementation5(self, device)
        self.compute_time_per_cycle = 0.0
        self.processing_current_cycle_data = threading.Lock()
        self.abortRequested = False

    def Reset(self) -> None:
        self.prms.SimulationStep = 0
        self.prms.SimulationTime = 0
        self.compute_time_per_cycle = 0.0

    def Prepare(self) -> None:
        self.abortRequested = False
        self.gpu.cuda_update_constants()

    def RequestAbort(self) -> None:
        self.abortRequested = True

    def UnlockCycleMutex(self) -> None:
        self.processing_current_cycle_data.release()

    def load_block(self, cells_x: int, cells_y: int, ind_y_above_floor: float = 0.2, grain_size: float = 0.05,
                   seed: int = 12345) -> None:
        """Synthetic stand-in for SnapshotManager::LoadRawPoints: builds the
        block, allocates, uploads, Reset and Prepare (snapshotmanager.cpp:186-286)."""
        n = 4 * cells_x * cells_y
        tmp = SimParams.copy(self.prms)
        make_block(tmp, cells_x, cells_y, ind_y_above_floor, grain_size, seed)
        C.memmove(C.byref(self.prms), C.byref(tmp), C.sizeof(SimParams))
        self.gpu.cuda_allocate_arrays(self.prms.GridTotal, n)
        make_block(self.prms, cells_x, cells_y, ind_y_above_floor, grain_size, seed, out=self.gpu.tmp_transfer_buffer)
        self.gpu.transfer_ponts_to_device()
        self.Reset()
        self.Prepare()

    def Step(self) -> bool:
        """One frame (model.cpp:11-47): reset the force bins, run substeps up
        to the next multiple of UpdateEveryNthStep, time them, copy the state
        back asynchronously. Returns False when the run should stop."""
        p = self.prms
        g = self.gpu
        g.cuda_reset_indenter_force_accumulator()
        timed = p.SimulationStep % (p.UpdateEveryNthStep * 2) == 0
        if timed:
            g.record_start()
        n = p.UpdateEveryNthStep - (p.SimulationStep % p.UpdateEveryNthStep)
        # the frame advances a copy: the consumer of the previous frame may
        # still read prms until the cycle lock is ours (model.cpp:32-45
        # updates them after taking it)
        nxt = SimParams.copy(p)
        g.run_substeps(nxt, n)
        if timed:
            g.record_stop()
        self.processing_current_cycle_data.acquire()
        p.SimulationStep, p.SimulationTime, p.indenter_x = nxt.SimulationStep, nxt.SimulationTime, nxt.indenter_x
        g.cuda_transfer_from_device()
        if not timed:
            self.compute_time_per_cycle = g.elapsed_ms() / p.UpdateEveryNthStep
        return p.SimulationTime < p.SimulationEndTime and not g.error_code


def repitch_soa(src: np.ndarray, src_pitch: int, n: int, dst: np.ndarray, dst_pitch: int) -> None:
    """Copies a particle SoA of n particles between pitches. Row 0 holds the
    crushed bytes at byte i and the grain ids at byte src_pitch + 2i
    (point.cpp:19-23), so it is moved field by field."""
    s = src[: src_pitch * N_PTS_ARRAYS].reshape(N_PTS_ARRAYS, src_pitch)
    d = dst[: dst_pitch * N_PTS_ARRAYS].reshape(N_PTS_ARRAYS, dst_pitch)
    d[1:, :n] = s[1:, :n]
    d[1:, n:] = 0
    sb = s[0].view(np.uint8)
    db = d[0].view(np.uint8)
    db[:] = 0
    db[:n] = sb[:n]
    db[dst_pitch: dst_pitch + 2 * n] = sb[src_pitch: src_pitch + 2 * n]


class SnapshotManager:
    """Mirror of icy::SnapshotManager (snapshotmanager.h:15-31) over the
    library's own HDF5 writer and reader."""

    directory_snapshots = "snapshots"
    directory_pq = "pq"

    def __init__(self, model: Optional["Model"] = None):
        self.model = model

    def SaveSnapshot(self, outputDirectory: str) -> str:
        """d%05d.h5 of the current frame (snapshotmanager.cpp:60-104);
        returns the path written."""
        m, g = self.model, self.model.gpu
        out = C.create_string_buffer(4096)
        _check(_lib().icm_save_snapshot(C.byref(m.prms), g.tmp_transfer_buffer.ctypes.data,
                                        g.host_side_indenter_force_accumulator.ctypes.data,
                                        os.fsencode(outputDirectory), out, len(out)))
        return out.value.decode()

    def ReadSnapshot(self, fileName: str) -> int:
        """Resumes from a snapshot (the reference's ReadSnapshot,
        snapshotmanager.cpp:145-184, is commented out): SimParams from the
        file with this run's device buffers (re-allocated when the sizes
        differ), the particle SoA uploaded, constants updated. Returns the
        frame number."""
        m, g = self.model, self.model.gpu
        tmp = SimParams()
        _check(_lib().icm_read_snapshot_params(os.fsencode(fileName), C.byref(tmp)))
        src_pitch = int(tmp.nPtsPitch)
        soa = np.empty(src_pitch * N_PTS_ARRAYS, dtype=np.float64)
        bins = np.empty(2 * tmp.n_indenter_subdivisions, dtype=np.float64)
        _check(_lib().icm_read_snapshot(os.fsencode(fileName), soa.ctypes.data, soa.size, bins.ctypes.data,
                                        bins.size))
        keep = {k: getattr(m.prms, k) for k in ("grid_array", "pts_array", "indenter_force_accumulator",
                                                 "nPtsPitch", "nGridPitch")}
        need_alloc = (not g.initialized or g.tmp_transfer_buffer is None or tmp.nPts > m.prms.nPts
                      or tmp.GridX * tmp.GridY > m.prms.GridX * m.prms.GridY
                      or tmp.n_indenter_subdivisions != m.prms.n_indenter_subdivisions)
        C.memmove(C.byref(m.prms), C.byref(tmp), C.sizeof(SimParams))
        if need_alloc:
            g.cuda_allocate_arrays(tmp.GridX * tmp.GridY, tmp.nPts)
        else:
            for k, v in keep.items():
                setattr(m.prms, k, v)
        repitch_soa(soa, src_pitch, int(tmp.nPts), g.tmp_transfer_buffer, int(m.prms.nPtsPitch))
        g.transfer_ponts_to_device()
        g.host_side_indenter_force_accumulator[:] = bins
        m.Prepare()
        return int(m.prms.SimulationStep // max(m.prms.UpdateEveryNthStep, 1))

    def LoadRawPoints(self, fileName: str) -> None:
        """snapshotmanager.cpp:186-286: reads the point cloud, allocates,
        uploads, Reset and Prepare."""
        m, g = self.model, self.model.gpu
        n = C.c_int(0)
        _check(_lib().icm_load_raw_points(C.byref(m.prms), os.fsencode(fileName), None, C.byref(n)))
        g.cuda_allocate_arrays(m.prms.GridTotal, n.value)
        _check(_lib().icm_load_raw_points(C.byref(m.prms), os.fsencode(fileName), g.tmp_transfer_buffer.ctypes.data,
                                          C.byref(n)))
        g.transfer_ponts_to_device()
        m.Reset()
        m.Prepare()

    def SavePQ(self, outputDirectory: str) -> str:
        """pq%05d.h5 of the current frame (snapshotmanager.cpp:14-56)."""
        m, g = self.model, self.model.gpu
        out = C.create_string_buffer(4096)
        _check(_lib().icm_save_pq(C.byref(m.prms), g.tmp_transfer_buffer.ctypes.data, os.fsencode(outputDirectory),
                                  out, len(out)))
        return out.value.decode()


def load_raw_points_host(prms: SimParams, fileName: str) -> np.ndarray:
    """LoadRawPoints into a host SoA only (no device): sets prms as the
    loader does and returns the 16 x pitch SoA (pitch from pitch_elems)."""
    n = C.c_int(0)
    _check(_lib().icm_load_raw_points(C.byref(prms), os.fsencode(fileName), None, C.byref(n)))
    prms.nPtsPitch = pitch_elems(n.value)
    out = np.zeros(prms.nPtsPitch * N_PTS_ARRAYS, dtype=np.float64)
    _check(_lib().icm_load_raw_points(C.byref(prms), os.fsencode(fileName), out.ctypes.data, C.byref(n)))
    return out


def save_snapshot_host(prms: SimParams, soa: np.ndarray, bins: np.ndarray, outputDirectory: str) -> str:
    """SaveSnapshot from host buffers (prms.nPtsPitch must describe soa)."""
    out = C.create_string_buffer(4096)
    _check(_lib().icm_save_snapshot(C.byref(prms), soa.ctypes.data, bins.ctypes.data, os.fsencode(outputDirectory),
                                    out, len(out)))
    return out.value.decode()


def read_snapshot_host(fileName: str):
    """(SimParams, SoA, bins) of a snapshot file, host only."""
    p = SimParams()
    _check(_lib().icm_read_snapshot_params(os.fsencode(fileName), C.byref(p)))
    soa = np.empty(int(p.nPtsPitch) * N_PTS_ARRAYS, dtype=np.float64)
    bins = np.empty(2 * p.n_indenter_subdivisions, dtype=np.float64)
    _check(_lib().icm_read_snapshot(os.fsencode(fileName), soa.ctypes.data, soa.size, bins.ctypes.data, bins.size))
    return p, soa, bins


def save_pq_host(prms: SimParams, soa: np.ndarray, outputDirectory: str) -> str:
    """SavePQ from a host SoA."""
    out = C.create_string_buffer(4096)
    _check(_lib().icm_save_pq(C.byref(prms), soa.ctypes.data, os.fsencode(outputDirectory), out, len(out)))
    return out.value.decode()


__all__ = ["SimParams", "BlockDesc", "GPU_Implementation5", "Model", "SoA", "make_block", "pitch_elems", "library",
           "SnapshotManager", "repitch_soa", "load_raw_points_host", "save_snapshot_host", "read_snapshot_host",
           "save_pq_host",
           "FORM_FP64_STEPWISE", "FORM_FP64", "FORM_FP32", "FORM_FP32_SURROGATE", "FORM_FP32_COMPENSATED", "FORM_NAMES", "TILE_VARIANTS", "LIB_PATH"]
