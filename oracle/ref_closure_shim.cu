// TEST INFRASTRUCTURE ONLY: the reference's CUDA scalar closure
// (src/reactiveTransport/reactiveClosureScalar.cuh, its plugin ABI
// reactive_closure_scalar_{create,run,destroy}_v1 of
// src/reactiveThermo/reactiveClosureAcceleration.h:37-42) compiled from the
// reference sources where they lie, for sm_100a, into oracle/_ref/. The GPU
// tests compare this library's ideal-gas closure with it; nothing in the
// product links or loads it.
#include <stdexcept>
#include <string>
#include "reactiveClosureScalar.cuh"
