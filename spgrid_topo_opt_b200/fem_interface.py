"""Python mirror of the solver's FEM interface and its binary wire format.

The reference defines the solver entry ``extern "C" void fem_solve(void *input,
void *output)`` together with the ``FEMInputs``/``FEMOutputs`` records and a
minimalist binary serializer (topo_opt/fem_interface.h:11,165-390 and
topo_opt/serialization.h:234-530).  This module restates those records and the
byte layout so that Python callers (tests, the benchmark, the autograd layer)
can build input blobs and read output blobs that are byte-compatible with the
C++ side:

* the blob starts with a ``size_t`` holding the total length (serialization.h:318-329);
* plain values are copied little-endian with their C++ size (int=4, double=8,
  bool=1, size_t=8) (serialization.h:366-398);
* ``std::vector`` and ``std::string`` carry a ``size_t`` element count first
  (serialization.h:462-483, 348-359);
* ``std::map`` carries a count followed by key/value pairs in key order
  (serialization.h:492-516);
* records are written field by field in the order of their ``io`` methods
  (fem_interface.h:182-190, 252-276, 373-381).

Block payloads are kept as numpy arrays: a ``BlockedGrid`` with ``n`` blocks is
``base`` (``int32[n,3]``) plus ``data`` (``float64[n,64]`` for scalars or
``float64[n,64,4]`` for the displacement grid), with the in-block index
``i*16 + j*4 + k`` (fem_interface.h:150-152).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

FEM_INTERFACE_VERSION_MAJOR = 3
FEM_INTERFACE_VERSION_MINOR = 1

_BLOCK_SIZE = 4
_BLOCK_VOLUME = _BLOCK_SIZE ** 3

FORCE_DTYPE = np.dtype([("coord", "<i4", (3,)), ("f", "<f8", (3,))])
DIRICHLET_DTYPE = np.dtype([("coord", "<i4", (3,)), ("axis", "<i4"), ("value", "<f8")])


class WireFormatError(ValueError):
    """Raised when a blob does not follow the FEM interface layout."""


# --------------------------------------------------------------------------
# Grids and records
# --------------------------------------------------------------------------
@dataclass
class BlockedGrid:
    """Sparse grid of 4x4x4 blocks (fem_interface.h:109-160)."""

    resolution: List[int] = field(default_factory=lambda: [0, 0, 0])
    base: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    data: np.ndarray = field(default_factory=lambda: np.zeros((0, _BLOCK_VOLUME), np.float64))

    @property
    def num_blocks(self) -> int:
        return int(self.base.shape[0])

    @staticmethod
    def index(i: int, j: int, k: int) -> int:
        """In-block linear index used by ``Block::get`` (fem_interface.h:150-152)."""
        return i * _BLOCK_SIZE * _BLOCK_SIZE + j * _BLOCK_SIZE + k


@dataclass
class KrylovSolverParameters:
    """Krylov parameters (fem_interface.h:84-96)."""

    tolerance: float = 1e-4
    max_iterations: int = 50
    restart_iterations: int = 0
    print_residuals: bool = False


@dataclass
class FEMInputs:
    """Solver inputs (fem_interface.h:226-363)."""

    version_major: int = FEM_INTERFACE_VERSION_MAJOR
    version_minor: int = FEM_INTERFACE_VERSION_MINOR
    extra_strings: Dict[str, str] = field(default_factory=dict)
    extra_ints: Dict[str, int] = field(default_factory=dict)
    extra_doubles: Dict[str, float] = field(default_factory=dict)
    resolution: List[int] = field(default_factory=lambda: [0, 0, 0])
    dx: float = 1.0
    krylov: KrylovSolverParameters = field(default_factory=KrylovSolverParameters)
    preserved_buffer_size: int = 0
    use_density_only: bool = True
    density: BlockedGrid = field(default_factory=BlockedGrid)
    mu: BlockedGrid = field(default_factory=BlockedGrid)
    lambda_: BlockedGrid = field(default_factory=BlockedGrid)
    global_mu: float = 0.0
    global_lambda: float = 0.0
    mg_level: int = 3
    explicit_mg_level: int = 0
    pre_and_post_smoothing_iter: int = 1
    bottom_smoothing_iter: int = 600
    jacobi_damping: float = 0.4
    caller_method: str = ""
    dirichlet_nodes: np.ndarray = field(default_factory=lambda: np.zeros(0, DIRICHLET_DTYPE))
    dirichlet_cells: np.ndarray = field(default_factory=lambda: np.zeros(0, DIRICHLET_DTYPE))
    forces: np.ndarray = field(default_factory=lambda: np.zeros(0, FORCE_DTYPE))

    # Accessors with the reference's defaults (fem_interface.h:278-328).
    def _int(self, key: str, default: int) -> int:
        return int(self.extra_ints.setdefault(key, default))

    def _double(self, key: str, default: float) -> float:
        return float(self.extra_doubles.setdefault(key, default))

    def keep_state(self) -> int:
        return self._int("keep_state", 0)

    def boundary_smoothing(self) -> int:
        return self._int("boundary_smoothing", 5)

    def forced_reuse(self) -> int:
        return self._int("forced_reuse", 0)

    def penalty(self) -> float:
        return self._double("penalty", 0.0)

    def minimum_stiffness(self) -> float:
        return self._double("minimum_stiffness", 0.0)

    def minimum_density(self) -> float:
        return self._double("minimum_density", 0.0)

    def stiffness_mapping(self, d):
        """SIMP map of fem_interface.h:343-353 (vectorised)."""
        p = self.penalty()
        if p:
            e_min = self.minimum_stiffness()
            return (1.0 - e_min) * np.power(np.maximum(self.minimum_density(), d), p) + e_min
        return d

    # Solver-state pointer split into two ints (fem_interface.h:193-209).
    def set_solver_state_ptr(self, ptr: int) -> None:
        self.extra_ints["state_ptr_lower"] = _as_int32(ptr & 0xFFFFFFFF)
        self.extra_ints["state_ptr_higher"] = _as_int32((ptr >> 32) & 0xFFFFFFFF)

    def get_solver_state_ptr(self) -> int:
        return _state_ptr(self.extra_ints)

    def preserve_output(self, num_active_blocks: int) -> None:
        """Size of the output buffer the caller reserves (fem_interface.h:445-454)."""
        self.preserved_buffer_size = (1 << 20) + num_active_blocks * (3 * 4 + 64 * 4 * 8)


@dataclass
class FEMOutputs:
    """Solver outputs (fem_interface.h:365-390)."""

    version_major: int = FEM_INTERFACE_VERSION_MAJOR
    version_minor: int = FEM_INTERFACE_VERSION_MINOR
    extra_strings: Dict[str, str] = field(default_factory=dict)
    extra_ints: Dict[str, int] = field(default_factory=dict)
    extra_doubles: Dict[str, float] = field(default_factory=dict)
    displacements: BlockedGrid = field(
        default_factory=lambda: BlockedGrid(data=np.zeros((0, _BLOCK_VOLUME, 4), np.float64)))
    residual_field: BlockedGrid = field(default_factory=BlockedGrid)
    info: str = ""
    residuals: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float64))
    error_code: int = 0
    success: bool = False

    def get_solver_state_ptr(self) -> int:
        return _state_ptr(self.extra_ints)

    def get_num_iterations(self) -> int:
        return int(self.residuals.shape[0])


def _as_int32(v: int) -> int:
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v & 0x80000000 else v


def _state_ptr(extra_ints: Dict[str, int]) -> int:
    if "state_ptr_lower" not in extra_ints:
        return 0
    lower = extra_ints["state_ptr_lower"] & 0xFFFFFFFF
    higher = extra_ints.get("state_ptr_higher", 0) & 0xFFFFFFFF
    return (higher << 32) + lower


# --------------------------------------------------------------------------
# Writer
# --------------------------------------------------------------------------
class _Writer:
    def __init__(self) -> None:
        self.parts: List[bytes] = [b"\0" * 8]  # placeholder for the total length

    def raw(self, b: bytes) -> None:
        self.parts.append(b)

    def i32(self, v: int) -> None:
        self.raw(struct.pack("<i", int(v)))

    def u64(self, v: int) -> None:
        self.raw(struct.pack("<Q", int(v)))

    def f64(self, v: float) -> None:
        self.raw(struct.pack("<d", float(v)))

    def boolean(self, v: bool) -> None:
        self.raw(struct.pack("<?", bool(v)))

    def string(self, s: str) -> None:
        b = s.encode("latin-1")
        self.u64(len(b))
        self.raw(b)

    def map_str_str(self, m: Dict[str, str]) -> None:
        self.u64(len(m))
        for k in sorted(m, key=lambda s: s.encode("latin-1")):
            self.string(k)
            self.string(m[k])

    def map_str_int(self, m: Dict[str, int]) -> None:
        self.u64(len(m))
        for k in sorted(m, key=lambda s: s.encode("latin-1")):
            self.string(k)
            self.i32(m[k])

    def map_str_double(self, m: Dict[str, float]) -> None:
        self.u64(len(m))
        for k in sorted(m, key=lambda s: s.encode("latin-1")):
            self.string(k)
            self.f64(m[k])

    def grid(self, g: BlockedGrid, vector: bool) -> None:
        for r in g.resolution:
            self.i32(r)
        n = g.num_blocks
        self.u64(n)
        if n == 0:
            return
        per = _BLOCK_VOLUME * (4 if vector else 1)
        rec = np.dtype([("base", "<i4", (3,)), ("data", "<f8", (per,))])
        arr = np.empty(n, rec)
        arr["base"] = np.asarray(g.base, np.int32).reshape(n, 3)
        arr["data"] = np.asarray(g.data, np.float64).reshape(n, per)
        self.raw(arr.tobytes())

    def records(self, arr: np.ndarray, dtype: np.dtype) -> None:
        arr = np.asarray(arr, dtype)
        self.u64(arr.shape[0])
        self.raw(arr.tobytes())

    def finish(self) -> bytes:
        total = sum(len(p) for p in self.parts)
        self.parts[0] = struct.pack("<Q", total)
        return b"".join(self.parts)


def _write_base(w: _Writer, obj) -> None:
    w.i32(obj.version_major)
    w.i32(obj.version_minor)
    w.map_str_str(obj.extra_strings)
    w.map_str_int(obj.extra_ints)
    w.map_str_double(obj.extra_doubles)


def serialize_inputs(p: FEMInputs) -> bytes:
    """Bytes of ``FEMInputs::io`` on a BinaryOutputSerializer (fem_interface.h:252-276)."""
    w = _Writer()
    _write_base(w, p)
    w.f64(p.dx)
    w.u64(p.preserved_buffer_size)
    w.boolean(p.use_density_only)
    if p.use_density_only:
        w.f64(p.global_mu)
        w.f64(p.global_lambda)
        w.grid(p.density, vector=False)
    else:
        w.grid(p.mu, vector=False)
        w.grid(p.lambda_, vector=False)
    w.i32(p.mg_level)
    w.i32(p.explicit_mg_level)
    w.i32(p.pre_and_post_smoothing_iter)
    w.i32(p.bottom_smoothing_iter)
    w.f64(p.jacobi_damping)
    for r in p.resolution:
        w.i32(r)
    w.records(p.forces, FORCE_DTYPE)
    w.records(p.dirichlet_nodes, DIRICHLET_DTYPE)
    w.records(p.dirichlet_cells, DIRICHLET_DTYPE)
    w.f64(p.krylov.tolerance)
    w.i32(p.krylov.max_iterations)
    w.i32(p.krylov.restart_iterations)
    w.boolean(p.krylov.print_residuals)
    w.string(p.caller_method)
    return w.finish()


def serialize_outputs(o: FEMOutputs) -> bytes:
    """Bytes of ``FEMOutputs::io`` (fem_interface.h:373-381)."""
    w = _Writer()
    _write_base(w, o)
    w.grid(o.displacements, vector=True)
    w.grid(o.residual_field, vector=False)
    w.string(o.info)
    w.u64(len(o.residuals))
    w.raw(np.asarray(o.residuals, "<f8").tobytes())
    w.i32(o.error_code)
    w.boolean(o.success)
    return w.finish()


# --------------------------------------------------------------------------
# Reader
# --------------------------------------------------------------------------
class _Reader:
    def __init__(self, blob, copy: bool = True) -> None:
        # any contiguous buffer (bytes, bytearray, a view of foreign memory) is
        # read in place; the grids are copied out of it unless copy is False,
        # in which case they are views that keep the blob alive
        self.copy = copy
        self.buf = memoryview(blob).cast("B")
        if len(self.buf) < 8:
            raise WireFormatError("blob shorter than its length header")
        (self.total,) = struct.unpack_from("<Q", self.buf, 0)
        if self.total > len(self.buf) or self.total < 8:
            raise WireFormatError(f"length header {self.total} does not fit a {len(self.buf)}-byte blob")
        self.head = 8

    def take(self, n: int) -> memoryview:
        if n < 0 or self.head + n > self.total:
            raise WireFormatError("blob truncated")
        v = self.buf[self.head:self.head + n]
        self.head += n
        return v

    def i32(self) -> int:
        return struct.unpack("<i", self.take(4))[0]

    def u64(self) -> int:
        return struct.unpack("<Q", self.take(8))[0]

    def f64(self) -> float:
        return struct.unpack("<d", self.take(8))[0]

    def boolean(self) -> bool:
        return bool(self.take(1)[0])

    def string(self) -> str:
        n = self.u64()
        return bytes(self.take(n)).decode("latin-1")

    def map(self, value_reader) -> dict:
        n = self.u64()
        out = {}
        for _ in range(n):
            k = self.string()
            out[k] = value_reader()
        return out

    def grid(self, vector: bool) -> BlockedGrid:
        res = [self.i32() for _ in range(3)]
        n = self.u64()
        per = _BLOCK_VOLUME * (4 if vector else 1)
        rec = np.dtype([("base", "<i4", (3,)), ("data", "<f8", (per,))])
        if n > (self.total - self.head) // rec.itemsize:
            raise WireFormatError("block count exceeds blob size")
        arr = np.frombuffer(self.take(n * rec.itemsize), rec, count=n)
        data = arr["data"].copy() if self.copy else arr["data"]
        data = data.reshape(n, _BLOCK_VOLUME, 4) if vector else data.reshape(n, _BLOCK_VOLUME)
        base = arr["base"].copy() if self.copy else arr["base"]
        if not self.copy:
            data.flags.writeable = False
            base.flags.writeable = False
        return BlockedGrid(resolution=res, base=base, data=data)

    def records(self, dtype: np.dtype) -> np.ndarray:
        n = self.u64()
        if n > (self.total - self.head) // dtype.itemsize:
            raise WireFormatError("record count exceeds blob size")
        return np.frombuffer(self.take(n * dtype.itemsize), dtype, count=n).copy()

    def done(self) -> None:
        if self.head != self.total:
            raise WireFormatError(f"{self.total - self.head} trailing bytes")


def _read_base(r: _Reader, obj) -> None:
    obj.version_major = r.i32()
    obj.version_minor = r.i32()
    if obj.version_major != FEM_INTERFACE_VERSION_MAJOR or obj.version_minor > FEM_INTERFACE_VERSION_MINOR:
        raise WireFormatError(f"unsupported interface version {obj.version_major}.{obj.version_minor}")
    obj.extra_strings = r.map(r.string)
    obj.extra_ints = r.map(r.i32)
    obj.extra_doubles = r.map(r.f64)


def deserialize_inputs(blob) -> FEMInputs:
    r = _Reader(blob)
    p = FEMInputs()
    _read_base(r, p)
    p.dx = r.f64()
    p.preserved_buffer_size = r.u64()
    p.use_density_only = r.boolean()
    if p.use_density_only:
        p.global_mu = r.f64()
        p.global_lambda = r.f64()
        p.density = r.grid(vector=False)
    else:
        p.mu = r.grid(vector=False)
        p.lambda_ = r.grid(vector=False)
    p.mg_level = r.i32()
    p.explicit_mg_level = r.i32()
    p.pre_and_post_smoothing_iter = r.i32()
    p.bottom_smoothing_iter = r.i32()
    p.jacobi_damping = r.f64()
    p.resolution = [r.i32() for _ in range(3)]
    p.forces = r.records(FORCE_DTYPE)
    p.dirichlet_nodes = r.records(DIRICHLET_DTYPE)
    p.dirichlet_cells = r.records(DIRICHLET_DTYPE)
    p.krylov = KrylovSolverParameters(r.f64(), r.i32(), r.i32(), r.boolean())
    p.caller_method = r.string()
    r.done()
    return p


def deserialize_outputs(blob, copy: bool = True) -> FEMOutputs:
    """Decode a FEMOutputs blob.  With copy=False the displacement and residual
    grids are read-only views into the blob (unaligned, record-strided), which
    stays alive as long as they do."""
    r = _Reader(blob, copy)
    o = FEMOutputs()
    _read_base(r, o)
    o.displacements = r.grid(vector=True)
    o.residual_field = r.grid(vector=False)
    o.info = r.string()
    n = r.u64()
    o.residuals = np.frombuffer(r.take(8 * n), "<f8").copy()
    o.error_code = r.i32()
    o.success = r.boolean()
    r.done()
    return o


def blob_length(blob) -> int:
    """Total length stored in a blob's header."""
    return struct.unpack_from("<Q", bytes(blob[:8]))[0]
