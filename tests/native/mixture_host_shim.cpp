// Test infrastructure only: the library's Peng-Robinson mixture evaluator
// (spuma-multiphysics_b200/csrc/pr_mixture.cuh, host and device code from one
// source) compiled for the host, so a CPU test can compare its arithmetic with
// the reference's own evaluator. The test builds this file into a temporary
// directory; nothing in the product links it.
#include "pr_mixture.cuh"

namespace {
void pack(const rb200::mix::Props& s, int ns, double* out, int* phase) {
    const double v[15] = {s.T, s.p, s.W, s.V, s.rho, s.e, s.h, s.s, s.cp, s.cv, s.alpha, s.kappaT, s.sound,
                          s.dpdT, s.dpdV};
    for (int i = 0; i < 15; ++i) out[i] = v[i];
    for (int k = 0; k < ns; ++k) out[15 + k] = s.mu[k];
    *phase = s.phase;
}
}  // namespace

extern "C" int mix_trho(const ReactiveB200Table* t, double T, double rho, const double* Y, int chem, double* out,
                        int* phase) {
    rb200::mix::Props s{};
    const int st = rb200::mix::trho(*t, T, rho, Y, chem != 0, s);
    if (st == 0) pack(s, t->ns, out, phase);
    return st;
}

extern "C" int mix_tp(const ReactiveB200Table* t, double T, double p, const double* Y, int choice, int chem,
                      double* out, int* phase) {
    rb200::mix::Props s{};
    const int st = rb200::mix::tp(*t, T, p, Y, choice, chem != 0, s);
    if (st == 0) pack(s, t->ns, out, phase);
    return st;
}

// The library's WALE PR scalar properties (wale_pr.cuh) for a batch of cells
// with the model image `model`: effective (ns per cell), cp, status per cell.
#include "wale_pr.cuh"
extern "C" void wale_pr_properties(const ReactiveB200HemModel* model, size_t count, const double* q,
                                   const ReactiveThermoState* states, const double* color, const double* jump,
                                   int enthalpies, double* effective, double* cp, int* status) {
    const int ns = model->ns;
    for (size_t c = 0; c < count; ++c) {
        double local[rb200::mix::kMaxNs] = {};
        double candidate = 0;
        status[c] = rb200::walepr::properties(*model, enthalpies ? q + c * ns : nullptr, states[c], color[c], jump[c],
                                              local, candidate, enthalpies != 0);
        cp[c] = candidate;
        for (int k = 0; k < ns; ++k) effective[c * ns + k] = local[k];
    }
}
