"""ctypes mirrors of the C-ABI structures in include/reactive_b200_types.h.

The layouts are the reference ABI's (src/reactiveTransport/reactiveTransport.h:10-23,
src/reactiveThermo/reactiveThermo.h:11-19, src/reactiveThermo/reactiveGpuHem.h:14-21,
src/reactiveThermo/reactiveDeviceFlash.h:39-53); the ctypes field lists are kept in
the same order as the reference's own ctypes harness
(tools/validate_reactive_transport.py:17-43) so a caller written against the
reference binds unchanged.
"""
import ctypes as C

import numpy as np


class Face(C.Structure):
    _fields_ = [(k, C.c_int64) for k in ("owner", "neighbour", "fixed")] + [
        ("normal", C.c_double * 3)] + [(k, C.c_double) for k in
        ("area", "distance", "ownerWeight")] + [("kind", C.c_int)]


class State(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("p", "T", "rho", "cv", "sound", "gasMass", "dilatation")]


class Config(C.Structure):
    _fields_ = [(k, C.c_size_t) for k in ("cells", "species", "variables", "faces", "fixed")] + [
        (k, C.c_double) for k in ("viscosity", "conductivity", "diffusivity", "waveFactor", "maxBytes")
    ] + [("mechanical", C.c_int)]


class Stats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in (
        "allocatedBytes", "uploadedBytes", "downloadedBytes", "kernelLaunches", "stages", "stepQueries")]


class Primitive(C.Structure):
    _fields_ = [("rho", C.c_double), ("u", C.c_double * 3)]


class Profile(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "conservedUploads", "conservedUploadBytes", "conservedDownloadBytes", "stateUploadBytes",
        "primitiveUploadBytes", "gasUploadBytes", "boundaryPartitions", "residentStages")]


class DeviceProfile(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "gasPropertyBuilds", "gasPropertyCells", "partitionUploadBytes", "thermoTableBytes",
        "gasStatusChecks", "cflFaceLaunches", "transportFaceLaunches", "faceWorkspaceBytes")]


class Token(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("attemptId", "stageId", "contentVersion")]


class OptionsV2(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32), ("bridgeCells", C.c_size_t),
                ("recomputeGas", C.c_int), ("physicalModelHash", C.c_char * 65)]


class MemoryV2(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "liveBytes", "peakBytes", "bridgeBytes", "conservedWorkspaceBytes", "gasWorkspaceBytes",
        "rhsWorkspaceBytes", "deviceToDeviceBytes", "synchronizations")]


class WaleOptions(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32), ("Cw", C.c_double)]


class WaleProfile(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32)] + [
        (n, C.c_uint64) for n in ("gradientBuilds", "viscosityBuilds", "cellsEvaluated", "workspaceBytes")]


class WaleScalarOptions(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32), ("turbulentPrandtl", C.c_double),
                ("turbulentSchmidt", C.c_double)]


class WaleScalarProfile(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32)] + [
        (n, C.c_uint64) for n in ("fieldUploads", "fieldUploadBytes", "workspaceBytes")]


class CapillaryOptions(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32), ("sigma", C.c_double),
                ("capillaryCfl", C.c_double), ("geometryEpsilon", C.c_double), ("condensableSpecies", C.c_int64)]


class CapillaryProfile(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32)] + [
        (n, C.c_uint64) for n in ("geometryBuilds", "geometryCells", "geometryKernels", "faceFluxBuilds",
                                  "colorUploadBytes", "geometryDownloadBytes", "capillaryWorkspaceBytes")]


class CapillaryResidentView(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32)] + [
        (n, C.c_void_p) for n in ("q", "energy", "seed", "capillary", "order", "output")] + [("count", C.c_size_t)]


class WalePrModel(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32), ("modelImage", C.c_void_p),
                ("modelBytes", C.c_size_t), ("physicalModelHash", C.c_char * 65), ("fixedCp", C.c_void_p),
                ("fixedSpeciesH", C.c_void_p)]


class WalePrEpoch(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32), ("nextConserved", Token),
                ("thermoVersion", C.c_uint64), ("geometryVersion", C.c_uint64), ("boundaryVersion", C.c_uint64),
                ("enthalpies", C.c_int)]


class WalePrProfile(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32)] + [
        (n, C.c_uint64) for n in ("builds", "cells", "kernels", "failures", "inputUploadBytes", "scratchBytes")] + [
        ("wallSeconds", C.c_double)]


class ThermoState(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "p", "T", "rho", "e", "entropy", "soundFrozen", "soundEquilibrium",
        "volumeResidual", "energyResidual", "chemicalResidual", "alphaGas")] + [
        ("alphaLiquid", C.c_double * 2), ("rhoGas", C.c_double), ("rhoLiquid", C.c_double * 2),
        ("liquidMass", C.c_double * 2), ("gasMass", C.c_double), ("cp", C.c_double), ("cv", C.c_double),
        ("activeLiquids", C.c_int), ("iterations", C.c_int)]


# numpy view of ReactiveThermoState so whole batches move without Python loops.
THERMO_DTYPE = np.dtype([
    ("p", "<f8"), ("T", "<f8"), ("rho", "<f8"), ("e", "<f8"), ("entropy", "<f8"),
    ("soundFrozen", "<f8"), ("soundEquilibrium", "<f8"), ("volumeResidual", "<f8"),
    ("energyResidual", "<f8"), ("chemicalResidual", "<f8"), ("alphaGas", "<f8"),
    ("alphaLiquid", "<f8", (2,)), ("rhoGas", "<f8"), ("rhoLiquid", "<f8", (2,)),
    ("liquidMass", "<f8", (2,)), ("gasMass", "<f8"), ("cp", "<f8"), ("cv", "<f8"),
    ("activeLiquids", "<i4"), ("iterations", "<i4")])

# ReactiveGpuHemOutputV1 (184 B) and ReactiveGpuHemCapillaryInputV2 (24 B)
HEM_OUTPUT_DTYPE = np.dtype([("state", THERMO_DTYPE), ("success", "<i4"), ("reserved", "<i4")])
CAPILLARY_DTYPE = np.dtype([("color", "<f8"), ("pressureJump", "<f8"), ("equilibrium", "<i4"), ("pad", "<i4")])
assert HEM_OUTPUT_DTYPE.itemsize == 184 and CAPILLARY_DTYPE.itemsize == 24
assert THERMO_DTYPE.itemsize == 176

STATE_DTYPE = np.dtype([(k, "<f8") for k in ("p", "T", "rho", "cv", "sound", "gasMass", "dilatation")])
FACE_DTYPE = np.dtype([("owner", "<i8"), ("neighbour", "<i8"), ("fixed", "<i8"), ("normal", "<f8", (3,)),
                       ("area", "<f8"), ("distance", "<f8"), ("ownerWeight", "<f8"), ("kind", "<i4"),
                       ("_pad", "<i4")])
assert FACE_DTYPE.itemsize == 80


class HemProfile(C.Structure):
    _fields_ = [("abiVersion", C.c_uint32), ("structBytes", C.c_uint32)] + [
        (n, C.c_uint64) for n in (
            "batches", "submitted", "succeeded", "cpuFallbacks", "deviceFailures",
            "phaseEvaluations", "residualEvaluations", "flashCandidates", "stableCandidates",
            "analyticJacobians", "finiteDifferenceJacobians", "transferBytes", "hostBytes",
            "deviceBytes")] + [(n, C.c_double) for n in ("wallSeconds", "kernelSeconds", "copySeconds")]


class NasaRegion(C.Structure):
    _fields_ = [("minimumTemperature", C.c_double), ("maximumTemperature", C.c_double),
                ("polynomial", C.c_int), ("coefficient", C.c_double * 9)]


class Species(C.Structure):
    _fields_ = [("molecularWeight", C.c_double), ("a", C.c_double), ("b", C.c_double),
                ("kappa", C.c_double), ("regionCount", C.c_int), ("regions", NasaRegion * 8)]


class Table(C.Structure):
    _fields_ = [("ns", C.c_int), ("refPressure", C.c_double), ("species", Species * 16),
                ("aBinary", (C.c_double * 16) * 16)]


class SolidModel(C.Structure):
    _fields_ = [("enabled", C.c_int), ("n", C.c_int)] + [
        (n, C.c_double) for n in ("Tmin", "Tmax", "Tref", "pref", "pmax", "molarVolume",
                                  "molecularWeight", "hRef", "sRef")] + [
        ("T", C.c_double * 64), ("cp", C.c_double * 64)]


class HemModel(C.Structure):
    _fields_ = [("phase", Table * 3), ("ns", C.c_int), ("nl", C.c_int), ("condensable", C.c_int * 2),
                ("boundaryRecovery", C.c_int), ("scalarRecovery", C.c_int), ("analyticJacobian", C.c_int),
                ("stableGasPrune", C.c_int), ("weights", C.c_double * 16), ("liquidTmin", C.c_double * 2),
                ("liquidTc", C.c_double * 2)] + [
        (n, C.c_double) for n in ("Tmin", "Tmax", "pmin", "pmax", "vtol", "etol", "mutol")] + [
        ("condensedKind", C.c_int * 2), ("enforceSpeciesTemperatureBounds", C.c_int),
        ("solid", SolidModel * 2)]


assert C.sizeof(Face) == 80 and C.sizeof(State) == 56 and C.sizeof(ThermoState) == 176
assert C.sizeof(HemModel) == 47448 and HemModel.stableGasPrune.offset == 45004
assert HemModel.weights.offset == 45008


def dptr(a):
    """Borrowed double* of a C-contiguous float64 numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))
