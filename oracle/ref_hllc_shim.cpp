// Test infrastructure: a C ABI over the reference's balanced-capillary face
// flux (src/reactiveInterface/reactiveBalancedCapillary.h:55-142) compiled for
// the host, called with no capillary terms (sigma = 0, zero surface stress),
// the plain HLLC core the transport's Faces functor applies
// (src/reactiveTransport/reactiveTransportKernels.h:357-417). Used only by the
// tests to pin oracle_hllc_face.
#include "reactiveBalancedCapillary.h"

extern "C" int ref_hllc_face(double rhoL, const double* uL, double pL, double aL, double EL, double rhoR,
                             const double* uR, double pR, double aR, double ER, const double* normal,
                             double* out) {
    ReactiveBalancedCapillary::State l{}, r{};
    l.rho = rhoL; l.pressure = pL; l.sound = aL; l.totalEnergy = EL; l.color = 0;
    r.rho = rhoR; r.pressure = pR; r.sound = aR; r.totalEnergy = ER; r.color = 0;
    ReactiveBalancedCapillary::Face f{};
    for (int d = 0; d < 3; ++d) { l.velocity[d] = uL[d]; r.velocity[d] = uR[d]; f.normal[d] = normal[d]; }
    ReactiveBalancedCapillary::Flux flux{};
    if (!ReactiveBalancedCapillary::faceFlux(l, r, f, flux)) return 0;
    out[0] = flux.contactSpeed; out[1] = flux.advectLeft; out[2] = flux.advectRight;
    out[3] = flux.pressureMomentum; out[4] = flux.pressureEnergy;
    return 1;
}
