// Batched Peng-Robinson mixture properties on the device: one thread per state
// through the host-and-device evaluator of pr_mixture.cuh.
#include "pr_mixture.cuh"
#include "common.cuh"
#include "../../include/reactive_b200_mixture.h"

#include <cstdio>
#include <exception>

namespace rb200 {
namespace {

constexpr int kMixOut = 15 + mix::kMaxNs;

__global__ void mixtureStates(const ReactiveB200Table* __restrict__ table, size_t count, const double* __restrict__ T,
                              const double* __restrict__ value, const double* __restrict__ Y, int mode, int choice,
                              double* __restrict__ out, int* __restrict__ status, int* __restrict__ phase) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < count; c += size_t(blockDim.x) * gridDim.x) {
        mix::Props s{};
        const double* y = Y + c * mix::kMaxNs;
        const int st = mode == 0 ? mix::trho(*table, T[c], value[c], y, true, s)
                                 : mix::tp(*table, T[c], value[c], y, choice, true, s);
        status[c] = st;
        if (st == mix::OK) {
            double* o = out + c * kMixOut;
            const double v[15] = {s.T, s.p, s.W, s.V, s.rho, s.e, s.h, s.s, s.cp, s.cv, s.alpha, s.kappaT,
                                  s.sound, s.dpdT, s.dpdV};
            for (int i = 0; i < 15; ++i) o[i] = v[i];
            for (int k = 0; k < mix::kMaxNs; ++k) o[15 + k] = k < table->ns ? s.mu[k] : 0.0;
            phase[c] = s.phase;
        }
    }
}

void fail(char* error, size_t size, const char* what) {
    if (error && size) std::snprintf(error, size, "%s", what);
}

}  // namespace
}  // namespace rb200

extern "C" int reactive_b200_mixture_properties_v3(const void* table, size_t count, const double* T,
                                                   const double* value, const double* Y, int mode, int choice,
                                                   double* out, int* status, int* phase, void* stream, char* error,
                                                   size_t size) {
    using namespace rb200;
    try {
        require(table && T && value && Y && out && status && phase, "Null mixture-property buffers");
        require(mode == 0 || mode == 1, "Mixture-property mode must be 0 (T, rho) or 1 (T, p)");
        require(choice >= 0 && choice <= 2, "Root choice must be 0 (auto), 1 (gas) or 2 (liquid)");
        if (!count) return 0;
        mixtureStates<<<gridFor(count, 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
            static_cast<const ReactiveB200Table*>(table), count, T, value, Y, mode, choice, out, status, phase);
        check(cudaGetLastError(), "mixtureStates");
        return 0;
    } catch (const std::exception& e) {
        fail(error, size, e.what());
        return 1;
    }
}
