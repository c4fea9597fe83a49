"""Python host wrapper of the reactive_gpu_hem_* ABI (the reference's GPU HEM
interface, src/reactiveThermo/reactiveGpuHem.h:40-84), driven with numpy host
arrays or torch device tensors."""
import ctypes as C

import numpy as np

from . import _abi as A, _lib
from .thermo_data import model_bytes, pure_model


class HemError(RuntimeError):
    pass


class GpuHem:
    """One HEM handle: a model image uploaded once and scratch for `capacity` cells."""

    def __init__(self, model=None, capacity=1, resident=False):
        self.lib = _lib.load()
        self.model = model if model is not None else pure_model()
        self.image = model_bytes(self.model) if not isinstance(self.model, (bytes, bytearray)) else bytes(self.model)
        err = C.create_string_buffer(1024)
        create = self.lib.reactive_gpu_hem_create_resident_v1 if resident else self.lib.reactive_gpu_hem_create_v1
        h = create(self.image, len(self.image), capacity, err, len(err))
        if not h:
            raise HemError(err.value.decode())
        self.handle = C.c_void_p(h)
        self.capacity = capacity

    def close(self):
        if getattr(self, "handle", None):
            self.lib.reactive_gpu_hem_destroy_v1(self.handle)
            self.handle = None

    __del__ = close

    @property
    def device_bytes(self):
        return self.lib.reactive_gpu_hem_device_bytes_v1(self.handle)

    def run(self, q, energy, states, success=None):
        """Flash host arrays in place: states (THERMO_DTYPE) are seeds in, results
        out for successful cells. success: an int32 array of the batch size to
        fill (pinned memory keeps its copy asynchronous), or None for a new one.
        Returns (success int32 array, profile)."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        energy = np.ascontiguousarray(energy, dtype=np.float64)
        assert states.dtype == A.THERMO_DTYPE and states.flags.c_contiguous
        n = len(energy)
        if success is None:
            success = np.zeros(n, dtype=np.int32)
        assert success.dtype == np.int32 and success.shape == (n,) and success.flags.c_contiguous
        prof = A.HemProfile(1, C.sizeof(A.HemProfile))
        err = C.create_string_buffer(1024)
        rc = self.lib.reactive_gpu_hem_run_v1(self.handle, A.dptr(q), A.dptr(energy), n,
                                              states.ctypes.data_as(C.c_void_p),
                                              success.ctypes.data_as(C.POINTER(C.c_int)), C.byref(prof), err, len(err))
        if rc:
            raise HemError(err.value.decode())
        return success, prof

    def run_capillary(self, q, energy, capillary, states, success=None):
        """The capillary batch (reactive_gpu_hem_run_v2) on host arrays: energy is the
        bulk internal energy density (kinetic and surface energy removed), capillary
        (CAPILLARY_DTYPE) each cell's color, pressure jump sigma*kappa and
        equilibrium flag (0: the frozen partition at the seed's liquid masses).
        states are seeds in, results out for successful cells.
        Returns (success int32 array, profile)."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        energy = np.ascontiguousarray(energy, dtype=np.float64)
        capillary = np.ascontiguousarray(capillary, dtype=A.CAPILLARY_DTYPE)
        assert states.dtype == A.THERMO_DTYPE and states.flags.c_contiguous
        n = len(energy)
        if success is None:
            success = np.zeros(n, dtype=np.int32)
        prof = A.HemProfile(1, C.sizeof(A.HemProfile))
        err = C.create_string_buffer(1024)
        rc = self.lib.reactive_gpu_hem_run_v2(self.handle, A.dptr(q), A.dptr(energy),
                                              capillary.ctypes.data_as(C.c_void_p), n,
                                              states.ctypes.data_as(C.c_void_p),
                                              success.ctypes.data_as(C.POINTER(C.c_int)), C.byref(prof), err, len(err))
        if rc:
            raise HemError(err.value.decode())
        return success, prof

    def initialize_capillary(self, q, energy, capillary, states, success=None):
        """The capillary primitive initialisation (reactive_gpu_hem_initialize_tp_v1)
        on host arrays, in place: q (cell-major) and energy become the normalised
        densities and their energy and states the initialised states, only if every
        cell succeeds. Returns (success int32 array, profile)."""
        assert q.dtype == np.float64 and q.flags.c_contiguous and energy.dtype == np.float64
        capillary = np.ascontiguousarray(capillary, dtype=A.CAPILLARY_DTYPE)
        n = len(energy)
        if success is None:
            success = np.zeros(n, dtype=np.int32)
        prof = A.HemProfile(1, C.sizeof(A.HemProfile))
        err = C.create_string_buffer(1024)
        rc = self.lib.reactive_gpu_hem_initialize_tp_v1(self.handle, A.dptr(q), A.dptr(energy),
                                                        capillary.ctypes.data_as(C.c_void_p), n,
                                                        states.ctypes.data_as(C.c_void_p),
                                                        success.ctypes.data_as(C.POINTER(C.c_int)), C.byref(prof),
                                                        err, len(err))
        if rc:
            raise HemError(err.value.decode())
        return success, prof

    def run_resident(self, q, energy, seed, capillary, order, count, output):
        """The device-resident batch (reactive_gpu_hem_run_resident_v1): device
        pointers or torch tensors indexed by cell; order[0..count) names the cells
        and each result goes to output[cell] (HEM_OUTPUT_DTYPE records).
        Returns the profile."""
        ptr = lambda t: None if t is None else (t if isinstance(t, int) else t.data_ptr())
        prof = A.HemProfile(1, C.sizeof(A.HemProfile))
        err = C.create_string_buffer(1024)
        rc = self.lib.reactive_gpu_hem_run_resident_v1(self.handle, ptr(q), ptr(energy), ptr(seed), ptr(capillary),
                                                       ptr(order), count, ptr(output), C.byref(prof), err, len(err))
        if rc:
            raise HemError(err.value.decode())
        return prof

    def run_device(self, conserved, stride, count, variables, seed, state=None, transport=None, success=None,
                   stream=0, per_cell=False):
        """Device batch: all arguments are device pointers (ints) or torch tensors.
        per_cell: the plain one-thread-per-cell form instead of the work-queue passes."""
        ptr = lambda t: 0 if t is None else (t if isinstance(t, int) else t.data_ptr())
        err = C.create_string_buffer(1024)
        rc = self.lib.reactive_gpu_hem_run_device_v3(self.handle, ptr(conserved), stride, count, variables,
                                                     ptr(seed), ptr(state), ptr(transport), ptr(success), None,
                                                     2 if per_cell else 0, stream, err, len(err))
        if rc:
            raise HemError(err.value.decode())

    def counters(self, stream=0):
        prof = A.HemProfile(1, C.sizeof(A.HemProfile))
        err = C.create_string_buffer(1024)
        if self.lib.reactive_gpu_hem_run_counters_v3(self.handle, C.byref(prof), stream, err, len(err)):
            raise HemError(err.value.decode())
        return prof
