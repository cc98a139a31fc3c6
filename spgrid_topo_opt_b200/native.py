"""ctypes binding of libspgrid_gpu_solver.so (the C ABI of include/spgrid_fem.h).

There is no CPU fallback: if the CUDA library is missing or no GPU is present,
the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from . import fem_interface as fi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspgrid_gpu_solver.so")

PRECISION_REFERENCE, PRECISION_FP64, PRECISION_MIXED, HOST_SETUP_ONLY = 0, 1, 2, 3
OP_KU, OP_RESIDUAL, OP_SMOOTH, OP_RESTRICT, OP_PROLONG, OP_STENCIL, OP_BOTTOM, OP_VCYCLE, OP_PACKED_RESIDUAL = range(9)

EXPORTED_SYMBOLS = ("fem_solve", "fem_solve_free", "sgs_create", "sgs_destroy", "sgs_last_error", "sgs_solve",
                    "sgs_residual_history", "sgs_displacements", "sgs_sensitivity", "sgs_level_count",
                    "sgs_level_blocks", "sgs_level_flags", "sgs_boundary_blocks", "sgs_apply", "sgs_level_stencils",
                    "sgs_codec_roundtrip", "sgs_time_op", "sgs_sensitivity_static", "sgs_set_density",
                    "sgs_filter_sensitivity", "sgs_oc_update", "sgs_design_set", "sgs_design_step",
                    "sgs_design_get", "sgs_band_create", "sgs_band_destroy", "sgs_band_last_error",
                    "sgs_band_set_density", "sgs_band_get_density", "sgs_band_set_fat", "sgs_band_update",
                    "sgs_band_maps", "sgs_band_attach", "sgs_band_session", "sgs_band_step", "sgs_render",
                    "sgs_band_render", "sgs_band_get_flags", "sgs_band_filter_voxels", "sgs_band_kill_below",
                    "sgs_band_threshold_density", "sgs_solution_size", "sgs_set_density_device",
                    "sgs_solution_device", "sgs_compliance_device", "sgs_sensitivity_device")

CELL_INSIDE, CELL_FORCE, CELL_FIXED = 1, 2, 4   # SGS_CELL_* (driver TopOptFlags bits 0-2)


class DesignParams(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("volume_fraction", C.c_double), ("step_limit", C.c_double),
                ("filter_size", C.c_double), ("minimum_density", C.c_double), ("fixed_density", C.c_double),
                ("smart_oc", C.c_int32), ("exclude_fixed", C.c_int32)]


class DesignResult(C.Structure):
    _fields_ = [("objective", C.c_double), ("change", C.c_double), ("lagrange", C.c_double),
                ("cg_iterations", C.c_int32), ("reserved", C.c_int32), ("solve_device_seconds", C.c_double),
                ("solve_seconds", C.c_double), ("step_seconds", C.c_double)]


class BandParams(C.Structure):
    _fields_ = [("minimum_density", C.c_double), ("active_threshold", C.c_double),
                ("fraction_to_keep", C.c_double), ("fat_margin", C.c_int32), ("connectivity_filtering", C.c_int32)]


class BandStats(C.Structure):
    _fields_ = [("container_blocks", C.c_int64), ("thin_before_pruning", C.c_int64), ("thin_blocks", C.c_int64),
                ("fat_blocks", C.c_int64), ("fatter_blocks", C.c_int64), ("components", C.c_int64),
                ("active_voxels", C.c_int64), ("device_seconds", C.c_double), ("fat_changed", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class VoxelStats(C.Structure):
    _fields_ = [("voxels", C.c_int64), ("components", C.c_int64), ("kept", C.c_int64), ("removed", C.c_int64),
                ("device_seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("mode", C.c_int32), ("frames", C.c_int32),
                ("threshold", C.c_float), ("extinction", C.c_float), ("slice", C.c_float), ("seed", C.c_uint32),
                ("camera", C.c_float * 12), ("reverse_mapping", C.c_int32), ("mirror", C.c_int32)]


def render_params(width: int, height: int, camera, mode: int = 0, frames: int = 1, threshold: float = 0.5,
                  extinction: float = 1.0, slice_: float = 0.99999, seed: int = 0,
                  reverse_mapping: bool = False, mirror: str = "") -> RenderParams:
    """mirror: any of "x", "y", "z" -- the volume shown mirrored across that far face."""
    cam = np.ascontiguousarray(camera, np.float32).reshape(12)
    bits = sum(1 << "xyz".index(a) for a in set(mirror))
    return RenderParams(width, height, mode, frames, threshold, extinction, slice_, seed,
                        (C.c_float * 12)(*cam.tolist()), int(reverse_mapping), bits)


def render(base: np.ndarray, density: np.ndarray, width: int, height: int, camera, **kw):
    """Render density blocks (FEMInputs layout) on the GPU (sgs_render): returns
    (uint32 image [height][width], volume resolution)."""
    b = np.ascontiguousarray(base, np.int32).reshape(-1, 3)
    d = np.ascontiguousarray(density, np.float64).reshape(-1, 64)
    p = render_params(width, height, camera, **kw)
    out = np.zeros((height, width), np.uint32)
    res = np.zeros(3, np.int32)
    rc = load().sgs_render(_ptr(b), b.shape[0], _ptr(d), C.byref(p), _ptr(out), _ptr(res))
    if rc != 0:
        raise SolverError(rc, "sgs_render failed")
    return out, res


def view_matrix(rx_deg: float = 0.0, ry_deg: float = 0.0, rz_deg: float = 0.0, tx: float = 0.0, ty: float = 0.0,
                tz: float = -4.0) -> np.ndarray:
    """The reference viewer's camera (misc/volume_renderer.cpp:124-146: glRotatef
    by -rx, -ry, -rz about x, y, z, then glTranslatef by -t, on the identity;
    default translation (0, 0, -4), :56) as the 3x4 row matrix the renderer
    takes."""
    def rot(axis, deg):
        a = np.deg2rad(deg)
        c, s = np.cos(a), np.sin(a)
        m = np.eye(4)
        i, j = [(1, 2), (2, 0), (0, 1)][axis]
        m[i, i], m[i, j], m[j, i], m[j, j] = c, -s, s, c
        return m
    t = np.eye(4)
    t[:3, 3] = [-tx, -ty, -tz]
    m = rot(0, -rx_deg) @ rot(1, -ry_deg) @ rot(2, -rz_deg) @ t
    return m[:3, :4].astype(np.float32).reshape(12)


def write_ppm(path: str, image: np.ndarray) -> None:
    """Save a packed RGBA image (row 0 at the bottom) as a binary PPM."""
    img = np.asarray(image, np.uint32)[::-1]
    rgb = np.stack([img & 0xFF, (img >> 8) & 0xFF, (img >> 16) & 0xFF], -1).astype(np.uint8)
    with open(path, "wb") as f:
        f.write(b"P6 %d %d 255\n" % (rgb.shape[1], rgb.shape[0]))
        f.write(rgb.tobytes())


class SolverError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[{code}] {message}")
        self.code = code


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("levels", C.c_int32), ("initial_residual", C.c_double),
                ("final_residual", C.c_double), ("setup_seconds", C.c_double), ("solve_seconds", C.c_double),
                ("launches_per_iteration", C.c_int64), ("dof", C.c_int64), ("bottom_unknowns", C.c_int64),
                ("solve_device_seconds", C.c_double), ("kernel_launches", C.c_int64), ("h2d_bytes", C.c_double),
                ("d2h_bytes", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load(build_if_missing: bool = False):
    """Load the CUDA library; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if build_if_missing:
            from .build import build
            build()
        else:
            raise ImportError(f"{LIB_PATH} is not built; run `python -m spgrid_topo_opt_b200.build`")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    L.fem_solve.argtypes = [P, P]
    L.fem_solve.restype = None
    L.fem_solve_free.argtypes = [P]
    L.sgs_create.argtypes = [P, C.c_int, C.POINTER(C.c_void_p), C.c_char_p, C.c_int]
    L.sgs_create.restype = C.c_int
    L.sgs_destroy.argtypes = [P]
    L.sgs_last_error.argtypes = [P]
    L.sgs_last_error.restype = C.c_char_p
    L.sgs_solve.argtypes = [P, C.c_double, C.c_int, C.POINTER(Stats)]
    L.sgs_residual_history.argtypes = [P, P, C.c_int]
    L.sgs_displacements.argtypes = [P, P]
    L.sgs_sensitivity.argtypes = [P, P, P, P]
    L.sgs_sensitivity.restype = C.c_double
    L.sgs_level_count.argtypes = [P]
    L.sgs_level_blocks.argtypes = [P, C.c_int, P]
    L.sgs_level_flags.argtypes = [P, C.c_int, P]
    L.sgs_boundary_blocks.argtypes = [P, C.c_int, P]
    L.sgs_apply.argtypes = [P, C.c_int, C.c_int, C.c_int, P, P, P]
    L.sgs_level_stencils.argtypes = [P, C.c_int, P, P]
    L.sgs_codec_roundtrip.argtypes = [P, C.c_int, C.POINTER(C.c_void_p)]
    L.sgs_time_op.argtypes = [P, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.sgs_sensitivity_static.argtypes = [P, P, P, P, P]
    L.sgs_sensitivity_static.restype = C.c_int
    L.sgs_set_density.argtypes = [P, P]
    L.sgs_filter_sensitivity.argtypes = [P, P, P, P, C.c_double]
    L.sgs_filter_sensitivity.restype = C.c_int
    L.sgs_oc_update.argtypes = [P, P, P, P, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.sgs_oc_update.restype = C.c_int
    L.sgs_design_set.argtypes = [P, P, P]
    L.sgs_design_set.restype = C.c_int
    L.sgs_design_step.argtypes = [P, C.POINTER(DesignParams), C.POINTER(DesignResult)]
    L.sgs_design_step.restype = C.c_int
    L.sgs_design_get.argtypes = [P, P]
    L.sgs_design_get.restype = C.c_int
    L.sgs_band_create.argtypes = [P, C.c_int64, P, P, P, C.POINTER(C.c_void_p), C.c_char_p, C.c_int]
    L.sgs_band_create.restype = C.c_int
    L.sgs_band_destroy.argtypes = [P]
    L.sgs_band_destroy.restype = None
    L.sgs_band_last_error.argtypes = [P]
    L.sgs_band_last_error.restype = C.c_char_p
    for name in ("sgs_band_set_density", "sgs_band_get_density", "sgs_band_set_fat"):
        getattr(L, name).argtypes = [P, P]
        getattr(L, name).restype = C.c_int
    L.sgs_band_update.argtypes = [P, C.POINTER(BandParams), C.POINTER(BandStats)]
    L.sgs_band_update.restype = C.c_int
    L.sgs_band_maps.argtypes = [P, P, P, P]
    L.sgs_band_maps.restype = C.c_int
    L.sgs_band_get_flags.argtypes = [P, P]
    L.sgs_band_get_flags.restype = C.c_int
    L.sgs_band_filter_voxels.argtypes = [P, C.POINTER(VoxelStats)]
    L.sgs_band_filter_voxels.restype = C.c_int
    L.sgs_band_kill_below.argtypes = [P, C.c_double, C.POINTER(C.c_int64)]
    L.sgs_band_kill_below.restype = C.c_int
    L.sgs_band_threshold_density.argtypes = [P, C.c_double, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_int64)]
    L.sgs_band_threshold_density.restype = C.c_int
    L.sgs_band_attach.argtypes = [P, P, P]
    L.sgs_band_attach.restype = C.c_int
    L.sgs_band_session.argtypes = [P, P, C.c_int, C.POINTER(C.c_void_p), C.c_char_p, C.c_int]
    L.sgs_band_session.restype = C.c_int
    L.sgs_band_step.argtypes = [P, P, C.POINTER(DesignParams), C.POINTER(DesignResult)]
    L.sgs_band_step.restype = C.c_int
    L.sgs_render.argtypes = [P, C.c_int64, P, C.POINTER(RenderParams), P, P]
    L.sgs_render.restype = C.c_int
    L.sgs_band_render.argtypes = [P, C.POINTER(RenderParams), P, P]
    L.sgs_band_render.restype = C.c_int
    L.sgs_solution_size.argtypes = [P]
    L.sgs_solution_size.restype = C.c_int64
    L.sgs_set_density_device.argtypes = [P, P, P]
    L.sgs_set_density_device.restype = C.c_int
    L.sgs_solution_device.argtypes = [P, P, P]
    L.sgs_solution_device.restype = C.c_int
    L.sgs_compliance_device.argtypes = [P, P, P]
    L.sgs_compliance_device.restype = C.c_int
    L.sgs_sensitivity_device.argtypes = [P, P, P, C.c_double, P, P, P]
    L.sgs_sensitivity_device.restype = C.c_int
    _lib = L
    return L


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def fem_solve_blob(blob: bytes) -> bytes:
    """Call the drop-in ``fem_solve`` entry with a serialized FEMInputs blob and
    return the serialized FEMOutputs blob (ownership handled as the reference's
    FEMInterface::run does, fem_interface.h:464-478)."""
    L = load()
    blob = bytes(blob)  # fem_solve only reads the input: pass the bytes object's own buffer
    out = C.c_void_p(0)
    L.fem_solve(C.cast(C.c_char_p(blob), C.c_void_p), C.cast(C.pointer(out), C.c_void_p))
    if not out.value:
        raise SolverError(11, "fem_solve returned no output blob")
    try:
        n = C.cast(out, C.POINTER(C.c_uint64))[0]
        data = C.string_at(out.value, n)
    finally:
        L.fem_solve_free(out)
    return data


class _LibraryBlob:
    """An output blob allocated by the library, exposed through the buffer
    protocol and released (fem_solve_free) when the last view of it is gone."""

    def __init__(self, address: int, size: int):
        self._address = address
        self._array = (C.c_char * size).from_address(address)

    def __buffer__(self, flags):
        return memoryview(self._array)

    def __release_buffer__(self, view):
        view.release()

    def __del__(self):
        if getattr(self, "_address", None):
            load().fem_solve_free(C.c_void_p(self._address))
            self._address = None


def fem_solve_outputs(blob: bytes):
    """``fem_solve`` on a serialized FEMInputs blob, returning the decoded
    FEMOutputs.  On Python 3.12+ the displacement field is a read-only view into
    the library's output blob, which is released when the arrays are (no copy);
    otherwise it is copied once out of the blob."""
    import sys
    from . import fem_interface as fi

    L = load()
    blob = bytes(blob)  # fem_solve only reads the input: pass the bytes object's own buffer
    out = C.c_void_p(0)
    L.fem_solve(C.cast(C.c_char_p(blob), C.c_void_p), C.cast(C.pointer(out), C.c_void_p))
    if not out.value:
        raise SolverError(11, "fem_solve returned no output blob")
    n = C.cast(out, C.POINTER(C.c_uint64))[0]
    if sys.version_info >= (3, 12):
        return fi.deserialize_outputs(_LibraryBlob(out.value, n), copy=False)
    try:
        return fi.deserialize_outputs((C.c_char * n).from_address(out.value))
    finally:
        L.fem_solve_free(out)


def codec_roundtrip(blob: bytes, which: int = 0) -> bytes:
    """Decode and re-encode a blob with the C++ codec (0 inputs, 1 outputs)."""
    L = load()
    buf = C.create_string_buffer(bytes(blob), len(blob))
    out = C.c_void_p(0)
    rc = L.sgs_codec_roundtrip(C.cast(buf, C.c_void_p), which, C.byref(out))
    if rc != 0:
        raise SolverError(rc, "codec rejected the blob")
    try:
        n = C.cast(out, C.POINTER(C.c_uint64))[0]
        return C.string_at(out.value, n)
    finally:
        L.fem_solve_free(out)


def fem_solve(inputs: fi.FEMInputs) -> fi.FEMOutputs:
    """Serialize, solve on the GPU, deserialize (FEMInterface::run equivalent)."""
    return fi.deserialize_outputs(fem_solve_blob(fi.serialize_inputs(inputs)))


class Session:
    """A problem resident on the GPU: set-up once, solve, read back."""

    def __init__(self, inputs, precision: int = PRECISION_REFERENCE):
        L = load()
        blob = inputs if isinstance(inputs, (bytes, bytearray)) else fi.serialize_inputs(inputs)
        self.inputs = inputs if not isinstance(inputs, (bytes, bytearray)) else fi.deserialize_inputs(blob)
        self._blob = C.create_string_buffer(bytes(blob), len(blob))
        h = C.c_void_p(0)
        err = C.create_string_buffer(512)
        rc = L.sgs_create(C.cast(self._blob, C.c_void_p), precision, C.byref(h), err, 512)
        if rc != 0:
            raise SolverError(rc, err.value.decode(errors="replace"))
        self.h = h
        self.precision = precision
        self.stats: Optional[dict] = None

    @classmethod
    def _adopt(cls, handle: C.c_void_p, precision: int) -> "Session":
        """Wrap a session the library built (no FEMInputs on the Python side)."""
        self = cls.__new__(cls)
        self.h = handle
        self.inputs = None
        self.precision = precision
        self.stats = None
        return self

    def close(self):
        if getattr(self, "h", None):
            load().sgs_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise SolverError(rc, load().sgs_last_error(self.h).decode(errors="replace"))

    def solve(self, tolerance: float = 0.0, max_iterations: int = 0) -> dict:
        st = Stats()
        self._check(load().sgs_solve(self.h, tolerance, max_iterations, C.byref(st)))
        self.stats = st.as_dict()
        return self.stats

    def history(self) -> np.ndarray:
        out = np.zeros(1024)
        n = load().sgs_residual_history(self.h, _ptr(out), 1024)
        return out[:min(n, 1024)].copy()

    def displacements(self) -> np.ndarray:
        nb = self.inputs.density.base.shape[0]
        out = np.zeros((nb, 64, 4))
        self._check(load().sgs_displacements(self.h, _ptr(out)))
        return out

    def sensitivity(self, density: Optional[np.ndarray] = None):
        rho = np.ascontiguousarray(self.inputs.density.data if density is None else density, np.float64)
        dc = np.zeros(rho.shape)
        se = np.zeros(rho.shape)
        obj = load().sgs_sensitivity(self.h, _ptr(rho), _ptr(dc), _ptr(se))
        if not np.isfinite(obj):
            raise SolverError(10, load().sgs_last_error(self.h).decode(errors="replace"))
        return obj, dc, se

    def filter_sensitivity(self, density: np.ndarray, dc0: np.ndarray, filter_size: float = 1.5) -> np.ndarray:
        """The driver's density-weighted sensitivity filter (Opt::smooth_dc,
        topo_opt/spgrid_topo_opt.cpp:527-579) on the GPU; dc0 is the gradient
        (the driver's sign, -dc of ``sensitivity``)."""
        rho = np.ascontiguousarray(density, np.float64)
        d0 = np.ascontiguousarray(dc0, np.float64)
        out = np.zeros(rho.shape)
        self._check(load().sgs_filter_sensitivity(self.h, _ptr(rho), _ptr(d0), _ptr(out), float(filter_size)))
        return out

    def oc_update(self, density: np.ndarray, dc0: np.ndarray, volume_fraction: float, step_limit: float = 0.2,
                  minimum_density: float = 0.0, fixed: Optional[np.ndarray] = None, fixed_density: float = 1.0,
                  smart_oc: bool = False, exclude_fixed: bool = True):
        """One optimality-criteria update (topo_opt/optimizer/optimality_criterion.cpp:19-145)
        on the GPU.  Returns (new density, Lagrange multiplier, largest change)."""
        rho = np.array(density, np.float64, copy=True, order="C")
        d0 = np.ascontiguousarray(dc0, np.float64)
        fx = None if fixed is None else np.ascontiguousarray(fixed, np.uint8)
        lag, chg = C.c_double(0), C.c_double(0)
        self._check(load().sgs_oc_update(self.h, _ptr(rho), _ptr(d0), None if fx is None else _ptr(fx),
                                         float(volume_fraction), float(step_limit), float(minimum_density),
                                         float(fixed_density), int(smart_oc), int(exclude_fixed), C.byref(lag),
                                         C.byref(chg)))
        return rho, lag.value, chg.value

    def design_set(self, density: np.ndarray, fixed: Optional[np.ndarray] = None) -> None:
        """Upload the densities of a device-resident optimizer loop (sgs_design_set)."""
        rho = np.ascontiguousarray(density, np.float64)
        fx = None if fixed is None else np.ascontiguousarray(fixed, np.uint8)
        self._design_keep = (rho, fx)
        self._check(load().sgs_design_set(self.h, _ptr(rho), None if fx is None else _ptr(fx)))

    def design_step(self, tolerance: float = 1e-6, volume_fraction: float = 0.1, step_limit: float = 0.2,
                    filter_size: float = 1.5, minimum_density: float = 0.0, fixed_density: float = 1.0,
                    smart_oc: bool = False, exclude_fixed: bool = True) -> dict:
        """One optimizer iteration on the GPU (sgs_design_step)."""
        p = DesignParams(tolerance, volume_fraction, step_limit, filter_size, minimum_density, fixed_density,
                         int(smart_oc), int(exclude_fixed))
        r = DesignResult()
        self._check(load().sgs_design_step(self.h, C.byref(p), C.byref(r)))
        return {k: getattr(r, k) for k, _ in DesignResult._fields_ if k != "reserved"}

    def design_get(self) -> np.ndarray:
        out = np.zeros(self.inputs.density.data.shape)
        self._check(load().sgs_design_get(self.h, _ptr(out)))
        return out

    def set_density(self, density: np.ndarray) -> None:
        """New densities for the same material pattern (operators are rebuilt)."""
        rho = np.ascontiguousarray(density, np.float64).reshape(-1, 64)
        if rho.shape[0] != self.inputs.density.base.shape[0]:
            raise ValueError("density must have one row of 64 values per input block")
        self._check(load().sgs_set_density(self.h, _ptr(rho)))
        self.inputs.density.data = rho.copy()

    # ---- device-resident calls (torch tensors on the session's device)
    @staticmethod
    def _stream():
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def set_density_device(self, rho) -> None:
        """New densities from a contiguous float64 CUDA tensor [nblocks, 64]."""
        self._check(load().sgs_set_density_device(self.h, C.c_void_p(rho.data_ptr()), self._stream()))

    def solution_size(self) -> int:
        return int(load().sgs_solution_size(self.h))

    def solution_device(self, out) -> None:
        """Copy the last solution (level-0 layout) into a float64 CUDA tensor."""
        self._check(load().sgs_solution_device(self.h, C.c_void_p(out.data_ptr()), self._stream()))

    def compliance_device(self, out) -> None:
        """out[0] = f.u of the last solve (a float64 CUDA tensor)."""
        self._check(load().sgs_compliance_device(self.h, C.c_void_p(out.data_ptr()), self._stream()))

    def sensitivity_device(self, u, rho, factor: float, scale, grad) -> None:
        """grad = factor * scale * p rho^(p-1) (1-Emin) u_e^T K0 u_e on the device;
        u a saved solution or None for the last solve, scale a one-element tensor or None."""
        self._check(load().sgs_sensitivity_device(
            self.h, None if u is None else C.c_void_p(u.data_ptr()), C.c_void_p(rho.data_ptr()), float(factor),
            None if scale is None else C.c_void_p(scale.data_ptr()), C.c_void_p(grad.data_ptr()), self._stream()))

    def time_op(self, op: int, reps: int = 20) -> float:
        """Average device milliseconds of a level-0 operator (0 the FP64 PCG
        matvec K*s, 1 residual, 2 smoothing sweep, 3 V-cycle, 4 K*u, 5 the
        residual on the tensor cores; 1, 2, 4 and 5 in the V-cycle's precision)
        on the resident data."""
        ms = C.c_double(0)
        self._check(load().sgs_time_op(self.h, op, reps, C.byref(ms)))
        return ms.value

    # ---- inspection / unit operators
    @property
    def levels(self) -> int:
        return load().sgs_level_count(self.h)

    def blocks(self, level: int) -> np.ndarray:
        n = load().sgs_level_blocks(self.h, level, None)
        out = np.zeros((n, 3), np.int32)
        load().sgs_level_blocks(self.h, level, _ptr(out))
        return out

    def flags(self, level: int) -> np.ndarray:
        n = self.blocks(level).shape[0]
        out = np.zeros(n * 128, np.uint32)
        load().sgs_level_flags(self.h, level, _ptr(out))
        return out

    def boundary_blocks(self, level: int) -> np.ndarray:
        n = load().sgs_boundary_blocks(self.h, level, None)
        out = np.zeros(n, np.int32)
        load().sgs_boundary_blocks(self.h, level, _ptr(out))
        return out

    def apply(self, op: int, level: int, x: np.ndarray, x2: Optional[np.ndarray] = None, arg: int = 0,
              out_level: Optional[int] = None) -> np.ndarray:
        ol = level if out_level is None else out_level
        n = self.blocks(ol).shape[0] * 128
        out = np.zeros((3, n))
        x = np.ascontiguousarray(x, np.float64)
        x2 = None if x2 is None else np.ascontiguousarray(x2, np.float64)
        self._check(load().sgs_apply(self.h, op, level, arg, _ptr(x), _ptr(x2), _ptr(out)))
        return out

    def stencils(self, level: int):
        n = self.blocks(level).shape[0] * 128
        out = np.zeros((n, 243))
        sp = np.zeros(n, np.uint32)
        self._check(load().sgs_level_stencils(self.h, level, _ptr(out), _ptr(sp)))
        return out, sp


class Band:
    """The optimizer driver's narrow band on the GPU: the container's 4x4x4
    blocks with per-cell flags (CELL_*) and densities, and the thin / fat /
    fatter page maps (include/spgrid_fem.h, sgs_band_*).  ``update`` runs the
    driver's update_thin_page_map, filter_isolated_blocks and
    update_fat_page_map (topo_opt/spgrid_topo_opt.cpp:92-241, 1404-1510);
    ``filter_voxels`` and ``threshold_and_kill`` its voxel-level clean-up
    (:1333-1344, 1512-1633).  ``flags`` is the host copy of the cell flags."""

    def __init__(self, base: np.ndarray, resolution, flags: np.ndarray, density: np.ndarray):
        L = load()
        self.base = np.ascontiguousarray(base, np.int32).reshape(-1, 3)
        self.n = self.base.shape[0]
        self.flags = np.ascontiguousarray(flags, np.uint8).reshape(self.n, 64)
        dens = np.ascontiguousarray(density, np.float64).reshape(self.n, 64)
        res = np.ascontiguousarray(resolution, np.int32).reshape(3)
        h = C.c_void_p(0)
        err = C.create_string_buffer(512)
        rc = L.sgs_band_create(_ptr(self.base), self.n, _ptr(res), _ptr(self.flags), _ptr(dens), C.byref(h), err, 512)
        if rc != 0:
            raise SolverError(rc, err.value.decode(errors="replace"))
        self.h = h
        self._initial_inside = (self.flags & CELL_INSIDE) != 0   # total_container_voxels counts these

    def close(self):
        if getattr(self, "h", None):
            load().sgs_band_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            raise SolverError(rc, load().sgs_band_last_error(self.h).decode(errors="replace"))

    def set_density(self, density: np.ndarray):
        d = np.ascontiguousarray(density, np.float64).reshape(self.n, 64)
        self._check(load().sgs_band_set_density(self.h, _ptr(d)))

    def density(self) -> np.ndarray:
        out = np.empty((self.n, 64))
        self._check(load().sgs_band_get_density(self.h, _ptr(out)))
        return out

    def set_fat(self, fat: np.ndarray):
        f = np.ascontiguousarray(np.asarray(fat) != 0, np.uint8)
        self._check(load().sgs_band_set_fat(self.h, _ptr(f)))

    def update(self, minimum_density: float = 0.0, active_threshold: float = 1e-6, fraction_to_keep: float = 1.0,
               fat_margin: int = 1, connectivity_filtering: bool = True) -> dict:
        p = BandParams(minimum_density, active_threshold, fraction_to_keep, fat_margin, int(connectivity_filtering))
        st = BandStats()
        self._check(load().sgs_band_update(self.h, C.byref(p), C.byref(st)))
        return st.as_dict()

    def maps(self):
        """(thin, fat, fatter) as bool[nblocks] in the container's block order."""
        t, f, ff = (np.zeros(self.n, np.uint8) for _ in range(3))
        self._check(load().sgs_band_maps(self.h, _ptr(t), _ptr(f), _ptr(ff)))
        return t != 0, f != 0, ff != 0

    def cell_flags(self) -> np.ndarray:
        out = np.empty((self.n, 64), np.uint8)
        self._check(load().sgs_band_get_flags(self.h, _ptr(out)))
        return out

    def filter_voxels(self) -> dict:
        """The driver's voxel_connectivity_filtering action, Opt::filter_isolated_voxels
        (topo_opt/spgrid_topo_opt.cpp:1512-1633): container cells of the thin
        blocks outside the one component above 30% leave the container with
        density 0 (sgs_band_filter_voxels)."""
        st = VoxelStats()
        self._check(load().sgs_band_filter_voxels(self.h, C.byref(st)))
        if st.removed:
            self.flags = self.cell_flags()
        return st.as_dict()

    def threshold_and_kill(self, threshold: float, **update) -> dict:
        """Opt::threshold_and_kill (topo_opt/spgrid_topo_opt.cpp:1333-1344):
        container cells below ``threshold`` leave the container, then the voxel
        filter and a page-map update without the block filter.  ``update`` takes
        the page-map settings of ``update``.  Returns the killed count and both
        stats.  As in the reference, the kill stays applied when the filter
        stops on an error."""
        k = C.c_int64(0)
        self._check(load().sgs_band_kill_below(self.h, float(threshold), C.byref(k)))
        if k.value:
            self.flags = self.cell_flags()
        vox = self.filter_voxels()
        maps = self.update(**dict(update, connectivity_filtering=False))
        return {"killed": int(k.value), "voxels": vox, "maps": maps}

    def threshold_density(self, volume_fraction: float = 0.1, threshold: Optional[float] = None):
        """Opt::threshold_density (topo_opt/spgrid_topo_opt.cpp:1756-1797): the
        cells of the fat blocks become 1 (density >= threshold, or fixed) or 0.
        Without ``threshold`` the reference's bisection finds the one that meets
        volume_fraction x the container voxels.  Returns (threshold, solid voxels)."""
        t = C.c_double(0)
        v = C.c_int64(0)
        self._check(load().sgs_band_threshold_density(self.h, float(volume_fraction),
                                                      -1.0 if threshold is None else float(threshold),
                                                      C.byref(t), C.byref(v)))
        return t.value, int(v.value)

    def packed_density(self) -> np.ndarray:
        """The densities of the session sgs_band_session packs from the maps
        (spgrid_topo_opt.cpp:1068-1160): the fatter blocks in container order,
        max(density, DBL_MIN) in the container cells of fat blocks, 0 elsewhere."""
        _, fat, fatter = self.maps()
        idx = np.nonzero(fatter)[0]
        rho = self.density()[idx]
        material = fat[idx][:, None] & ((self.flags[idx] & CELL_INSIDE) != 0)
        return np.where(material, np.maximum(rho, np.finfo(np.float64).tiny), 0.0)

    def threshold_and_compute_objective(self, template, volume_fraction: float = 0.1,
                                        threshold: Optional[float] = None, precision: int = PRECISION_MIXED,
                                        tolerance: float = 0.0) -> dict:
        """The driver's threshold_and_compute_objective action
        (topo_opt/spgrid_topo_opt.cpp:839-864): threshold the design (bisection
        when no threshold is given, the volume then reported as volume_fraction x
        the container voxels; with a threshold, its solid count), solve the
        packed design and evaluate the compliance objective."""
        t, solid = self.threshold_density(volume_fraction, threshold)
        vol = float(solid) if threshold is not None else float(volume_fraction * int(
            np.count_nonzero(self._initial_inside)))
        with self.session(template, precision) as s:
            st = s.solve(tolerance)
            obj, _, _ = s.sensitivity(self.packed_density())
        return {"objective": obj, "volume": vol, "threshold": t, "solid_voxels": solid,
                "cg_iterations": st["iterations"]}

    def attach(self, session: "Session", container_block: np.ndarray):
        """Bind a session built from this band's fatter blocks: its input block i
        is container block ``container_block[i]`` (sgs_band_attach)."""
        idx = np.ascontiguousarray(container_block, np.int64)
        self._check(load().sgs_band_attach(self.h, session.h, _ptr(idx)))

    def step(self, session: "Session", tolerance: float = 1e-6, volume_fraction: float = 0.1,
             step_limit: float = 0.2, filter_size: float = 1.5, minimum_density: float = 0.0,
             fixed_density: float = 1.0, smart_oc: bool = False, exclude_fixed: bool = True) -> dict:
        """One driver iteration on the band (sgs_band_step)."""
        p = DesignParams(tolerance, volume_fraction, step_limit, filter_size, minimum_density, fixed_density,
                         int(smart_oc), int(exclude_fixed))
        r = DesignResult()
        self._check(load().sgs_band_step(self.h, session.h, C.byref(p), C.byref(r)))
        return {k: getattr(r, k) for k, _ in DesignResult._fields_ if k != "reserved"}

    def session(self, template, precision: int = PRECISION_MIXED) -> "Session":
        """A session packed from the band's fatter blocks and densities, already
        attached (sgs_band_session); ``template`` gives the solver settings and
        boundary conditions (FEMInputs or its blob; its density grid is ignored)."""
        blob = template if isinstance(template, (bytes, bytearray)) else fi.serialize_inputs(template)
        buf = C.create_string_buffer(bytes(blob), len(blob))
        h = C.c_void_p(0)
        err = C.create_string_buffer(512)
        rc = load().sgs_band_session(self.h, C.cast(buf, C.c_void_p), precision, C.byref(h), err, 512)
        if rc != 0:
            raise SolverError(rc, err.value.decode(errors="replace"))
        return Session._adopt(h, precision)

    def render(self, width: int, height: int, camera, **kw):
        """Render the band's current densities (sgs_band_render)."""
        p = render_params(width, height, camera, **kw)
        out = np.zeros((height, width), np.uint32)
        res = np.zeros(3, np.int32)
        self._check(load().sgs_band_render(self.h, C.byref(p), _ptr(out), _ptr(res)))
        return out, res
