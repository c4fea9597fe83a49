// Test infrastructure only: a C-ABI shim that runs the REFERENCE project's own
// allocation-free UV flash (src/reactiveThermo/reactiveDeviceFlash.h) on the
// host, so parity tests and the CPU baseline can call it through ctypes.
// Nothing in the product links or loads this file; it is compiled by
// oracle/Makefile from the reference headers where they lie, with output only
// in oracle/_ref/.
//
// Entry points:
//   ref_flash_model_bytes        sizeof(ReactiveDeviceFlash::Model) (47,448)
//   ref_flash_valid_model        ReactiveDeviceFlash::validModel (reactiveDeviceFlash.h:80)
//   ref_flash_recover            ReactiveDeviceFlash::recover per cell
//                                (reactiveDeviceFlash.h:564) with the pure-liquid
//                                reported-phase cache that the reference CUDA kernel
//                                builds (reactiveGpuHem.cuh:31-36), threads optional
//   ref_flash_recover_capillary  ReactiveDeviceFlash::recoverCapillary per cell
//                                (reactiveDeviceFlash.h:572-588): per-cell color,
//                                pressure jump and equilibrium flag; status per cell
//   ref_flash_initialize_tp      ReactiveDeviceFlash::initializeCapillaryTP per cell
//                                (reactiveDeviceFlash.h:589-613)
//   ref_wale_pr_evaluate         ReactiveDeviceWalePr::evaluate per cell
//                                (reactiveDeviceWalePr.h:20-103): the phase-aware cp
//                                and effective species enthalpies at accepted states
//   ref_pr_evaluate_tp / _trho   ReactiveDevicePR::evaluateTPTrusted / evaluateTrhoTrusted
//                                (reactiveDevicePR.h:575, :474) for EOS unit checks
//   ref_pr_mix_tp / _trho        the same for a mixture table with mass fractions Y
#include "reactiveDeviceFlash.h"
#include "reactiveDeviceWalePr.h"
#include <cstring>
#include <thread>
#include <vector>
#include <atomic>

namespace {
using Model = ReactiveDeviceFlash::Model;
using Cache = ReactiveDevicePRPurePhaseCache::PureReportedPhaseCache;
}

extern "C" {

size_t ref_flash_model_bytes(void) { return sizeof(Model); }

int ref_flash_valid_model(const void* image) {
    Model m;
    std::memcpy(&m, image, sizeof(m));
    return ReactiveDeviceFlash::validModel(m) ? 1 : 0;
}

// counters: 7 uint64 per cell (phases, residuals, candidates, stable, failures,
// analyticJacobians, finiteDifferenceJacobians); may be null.
int ref_flash_recover(const void* image, size_t count, const double* q, const double* energy,
                      const ReactiveThermoState* guess, ReactiveThermoState* out, int* success,
                      uint64_t* counters, int useCache, int threads) {
    Model* m = new Model;
    std::memcpy(m, image, sizeof(Model));
    if (!ReactiveDeviceFlash::validModel(*m)) { delete m; return 1; }
    Cache cache[2]{};
    if (useCache)
        for (int i = 0; i < m->nl && i < 2; ++i)
            ReactiveDevicePRPurePhaseCache::buildPureReportedPhaseCache(m->phase[i + 1], cache[i]);
    const int ns = m->ns;
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const size_t c = next.fetch_add(1);
            if (c >= count) break;
            ReactiveDeviceFlash::Input in{};
            for (int k = 0; k < ns; ++k) in.q[k] = q[c * ns + k];
            in.energy = energy[c];
            in.guess = guess[c];
            const ReactiveDeviceFlash::Output o =
                ReactiveDeviceFlash::recover(*m, in, useCache ? cache : nullptr);
            out[c] = o.success ? o.state : guess[c];
            success[c] = o.success;
            if (counters) {
                uint64_t* k = counters + 7 * c;
                k[0] = o.counters.phases; k[1] = o.counters.residuals; k[2] = o.counters.candidates;
                k[3] = o.counters.stable; k[4] = o.counters.failures;
                k[5] = o.counters.analyticJacobians; k[6] = o.counters.finiteDifferenceJacobians;
            }
        }
    };
    if (threads <= 1) worker();
    else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
    }
    delete m;
    return 0;
}

// The capillary batch: color[c], jump[c], equilibrium[c] per cell; a failed
// cell keeps its seed in out; status[c] is the reference's Output.status
// (0 success, 1 no candidate, 2 invalid capillary input).
int ref_flash_recover_capillary(const void* image, size_t count, const double* q, const double* energy,
                                const ReactiveThermoState* guess, const double* color, const double* jump,
                                const int* equilibrium, ReactiveThermoState* out, int* success, int* status,
                                uint64_t* counters, int threads) {
    Model* m = new Model;
    std::memcpy(m, image, sizeof(Model));
    if (!ReactiveDeviceFlash::validModel(*m)) { delete m; return 1; }
    Cache cache[2]{};
    for (int i = 0; i < m->nl && i < 2; ++i)
        ReactiveDevicePRPurePhaseCache::buildPureReportedPhaseCache(m->phase[i + 1], cache[i]);
    const int ns = m->ns;
    std::atomic<size_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const size_t c = next.fetch_add(1);
            if (c >= count) break;
            ReactiveDeviceFlash::Input in{};
            for (int k = 0; k < ns; ++k) in.q[k] = q[c * ns + k];
            in.energy = energy[c];
            in.guess = guess[c];
            const ReactiveDeviceFlash::Output o =
                ReactiveDeviceFlash::recoverCapillary(*m, in, color[c], jump[c], equilibrium[c] != 0, cache);
            out[c] = o.success ? o.state : guess[c];
            success[c] = o.success;
            status[c] = o.status;
            if (counters) {
                uint64_t* k = counters + 7 * c;
                k[0] = o.counters.phases; k[1] = o.counters.residuals; k[2] = o.counters.candidates;
                k[3] = o.counters.stable; k[4] = o.counters.failures;
                k[5] = o.counters.analyticJacobians; k[6] = o.counters.finiteDifferenceJacobians;
            }
        }
    };
    if (threads <= 1) worker();
    else {
        std::vector<std::thread> pool;
        for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
        for (auto& t : pool) t.join();
    }
    delete m;
    return 0;
}

// The capillary primitive initialisation (initializeCapillaryTP,
// reactiveDeviceFlash.h:589-613) per cell: q and energy are replaced by the
// normalised densities where a cell succeeds; out receives the state.
int ref_flash_initialize_tp(const void* image, size_t count, double* q, double* energy,
                            const ReactiveThermoState* guess, const double* color, const double* jump,
                            ReactiveThermoState* out, int* success, int* status) {
    Model* m = new Model;
    std::memcpy(m, image, sizeof(Model));
    if (!ReactiveDeviceFlash::validModel(*m)) { delete m; return 1; }
    Cache cache[2]{};
    for (int i = 0; i < m->nl && i < 2; ++i)
        ReactiveDevicePRPurePhaseCache::buildPureReportedPhaseCache(m->phase[i + 1], cache[i]);
    const int ns = m->ns;
    for (size_t c = 0; c < count; ++c) {
        ReactiveDeviceFlash::Input in{};
        for (int k = 0; k < ns; ++k) in.q[k] = q[c * ns + k];
        in.energy = energy[c];
        in.guess = guess[c];
        double mass[ReactiveDeviceFlash::maxSpecies]{};
        double e = energy[c];
        const ReactiveDeviceFlash::Output o =
            ReactiveDeviceFlash::initializeCapillaryTP(*m, in, color[c], jump[c], mass, e, cache);
        out[c] = o.state;
        success[c] = o.success;
        status[c] = o.status;
        if (o.success) {
            for (int k = 0; k < ns; ++k) q[c * ns + k] = mass[k];
            energy[c] = e;
        }
    }
    delete m;
    return 0;
}

// The WALE PR scalar properties per cell: total species densities q (ns per
// cell), the accepted state, color and jump; effective (ns per cell) and cp out,
// status[c] the reference's Status (0 success).
int ref_wale_pr_evaluate(const void* image, size_t count, const double* q, const ReactiveThermoState* states,
                         const double* color, const double* jump, int enthalpies, double* effective, double* cp,
                         int* status) {
    Model* m = new Model;
    std::memcpy(m, image, sizeof(Model));
    if (!ReactiveDeviceFlash::validModel(*m)) { delete m; return 1; }
    const int ns = m->ns;
    for (size_t c = 0; c < count; ++c) {
        double local[ReactiveDeviceFlash::maxSpecies]{};
        double candidate = 0;
        status[c] = int(ReactiveDeviceWalePr::evaluate(*m, enthalpies ? q + c * ns : nullptr, states[c], color[c],
                                                       jump[c], local, candidate, enthalpies != 0));
        cp[c] = candidate;
        for (int k = 0; k < ns; ++k) effective[c * ns + k] = local[k];
    }
    delete m;
    return 0;
}

// out[0..15]: T p W V rho e h s cp cv alpha kappaT sound dpdT dpdV mu0 ; phaseOut: phase
static void packState(const ReactiveDevicePR::State& s, double* out, int* phaseOut) {
    const double v[16] = {s.T, s.p, s.W, s.V, s.rho, s.e, s.h, s.s, s.cp, s.cv,
                          s.alpha, s.kappaT, s.sound, s.dpdT, s.dpdV, s.mu[0]};
    std::memcpy(out, v, sizeof(v));
    if (phaseOut) *phaseOut = s.phase;
}

int ref_pr_evaluate_tp(const void* image, int table, double T, double p, int choice,
                       int chemical, double* out, int* phase) {
    Model* m = new Model;
    std::memcpy(m, image, sizeof(Model));
    double Y[ReactiveDeviceFlash::maxSpecies]{};
    Y[0] = 1.0;
    ReactiveDevicePR::State s{};
    const auto st = ReactiveDevicePR::evaluateTPTrusted(m->phase[table], T, p, Y,
        static_cast<ReactiveDevicePR::RootChoice>(choice), s, chemical != 0);
    if (st == ReactiveDevicePR::Status::Success) packState(s, out, phase);
    delete m;
    return static_cast<int>(st);
}

int ref_pr_evaluate_trho(const void* image, int table, double T, double rho, int chemical,
                         double* out, int* phase) {
    Model* m = new Model;
    std::memcpy(m, image, sizeof(Model));
    double Y[ReactiveDeviceFlash::maxSpecies]{};
    Y[0] = 1.0;
    ReactiveDevicePR::State s{};
    const auto st = ReactiveDevicePR::evaluateTrhoTrusted(m->phase[table], T, rho, Y, s, chemical != 0);
    if (st == ReactiveDevicePR::Status::Success) packState(s, out, phase);
    delete m;
    return static_cast<int>(st);
}

// Mixture forms with mass fractions Y (table's ns entries); out receives the 15
// properties of packState and then mu[0..ns).
static void packMix(const ReactiveDevicePR::State& s, int ns, double* out, int* phaseOut) {
    const double v[15] = {s.T, s.p, s.W, s.V, s.rho, s.e, s.h, s.s, s.cp, s.cv,
                          s.alpha, s.kappaT, s.sound, s.dpdT, s.dpdV};
    std::memcpy(out, v, sizeof(v));
    for (int k = 0; k < ns; ++k) out[15 + k] = s.mu[k];
    if (phaseOut) *phaseOut = s.phase;
}

int ref_pr_mix_trho(const void* image, int table, double T, double rho, const double* Yin, int chemical,
                    double* out, int* phase) {
    Model* m = new Model;
    std::memcpy(m, image, sizeof(Model));
    double Y[ReactiveDeviceFlash::maxSpecies]{};
    const int ns = m->phase[table].ns;
    for (int k = 0; k < ns; ++k) Y[k] = Yin[k];
    ReactiveDevicePR::State s{};
    const auto st = ReactiveDevicePR::evaluateTrhoTrusted(m->phase[table], T, rho, Y, s, chemical != 0);
    if (st == ReactiveDevicePR::Status::Success) packMix(s, ns, out, phase);
    delete m;
    return static_cast<int>(st);
}

int ref_pr_mix_tp(const void* image, int table, double T, double p, const double* Yin, int choice, int chemical,
                  double* out, int* phase) {
    Model* m = new Model;
    std::memcpy(m, image, sizeof(Model));
    double Y[ReactiveDeviceFlash::maxSpecies]{};
    const int ns = m->phase[table].ns;
    for (int k = 0; k < ns; ++k) Y[k] = Yin[k];
    ReactiveDevicePR::State s{};
    const auto st = ReactiveDevicePR::evaluateTPTrusted(m->phase[table], T, p, Y,
        static_cast<ReactiveDevicePR::RootChoice>(choice), s, chemical != 0);
    if (st == ReactiveDevicePR::Status::Success) packMix(s, ns, out, phase);
    delete m;
    return static_cast<int>(st);
}

}  // extern "C"
