"""Species property data and the HEM model image for the pure-N2O Peng-Robinson case.

The numbers are physical input data of the reference's N2O case, restated here:
* Peng-Robinson a [Pa m^6/kmol^2], b [m^3/kmol] and acentric factor, and the NASA9
  ideal-gas polynomials with their temperature ranges, from
  examples/impinging-n2o-supercooled/cold-pr-148K.yaml:172-231 (N2O), :52-111 (N2),
  :112-171 (O2) and :232-282 (IC3H7OH); molecular weights from the elements
  (N 14.007, O 15.999, C 12.011, H 1.008);
* flash bounds and tolerances from examples/impinging-n2o-supercooled/cold-pr-148K-config.yaml:1-19;
* molecular weight 44.013 kg/kmol, the value the reference records for N2O
  (results/real-fluid-v2-20260919/physical-model-manifest.json:147);
* reference pressure one standard atmosphere (the thermodynamic library default that
  the reference exporter copies, src/reactiveThermo/reactiveDevicePRExport.h:37).

The model image is the reference's 47,448-byte POD layout
(src/reactiveThermo/reactiveDeviceFlash.h:39-53); field meanings follow the
reference exporter (src/reactiveThermo/reactiveDevicePRExport.h:80-100 for kappa and
the geometric a_ij mixing rule).
"""
import ctypes as C
import math

import numpy as np

from ._abi import HemModel

GAS_CONSTANT = 8314.46261815324  # J/(kmol K), CODATA 2018
ONE_ATM = 101325.0
OMEGA_A = 4.5723552892138218e-1
OMEGA_B = 7.77960739038885e-2

N2O = dict(
    name="N2O", W=44.013, a=417972.1865083438, b=0.02763390066995578, omega=0.1613,
    ranges=[148.0, 182.34, 200.0, 1420.0, 3500.0],
    nasa9=[
        [-13883.483314218653, 400.2145375936049, 0.08987442809300043, -0.002575847027809755,
         0.00015894592824637003, -5.833630345245842e-07, 6.961726174507204e-10,
         6995.331413063375, 24.693976510805115],
        [0.0, 0.0, 4.796459403683242, -0.03064976304265226, 0.000248176450083356,
         -7.193439839786354e-07, 7.637795272607834e-10, 8617.974553201218, 2.097742156376054],
        [0.0, 0.0, 2.51620681, 0.00916990584, -7.8942084e-06, 3.42198245e-09,
         -5.84582078e-13, 8720.2997, 9.7150932],
        [0.0, 0.0, 4.85543722, 0.0025805244, -9.33594196e-07, 1.54088463e-10,
         -9.24862861e-15, 8055.95827, -2.39060855],
    ])

N2 = dict(
    name="N2", W=28.014, a=148227.8749500853, b=0.02403707313054656, omega=0.0372,
    ranges=[148.0, 182.34, 200.0, 1050.0, 3500.0],
    nasa9=[
        [98.29709685176373, -3.927219570926414, 3.5657235265591836, -0.0005864923434821304,
         2.999170859129467e-06, -8.169508775555017e-09, 9.359447755361056e-12,
         -1028.6313331407114, 2.811951852573376],
        [0.0, 0.0, 3.517433744475874, -8.456160143098416e-05, 7.709235665872965e-07,
         -3.002427186776785e-09, 4.451086162653223e-12, -1045.881160054519, 3.01983695239548],
        [0.0, 0.0, 3.73100682, -0.0018315973, 4.32324662e-06, -3.04378151e-09,
         7.46071562e-13, -1062.87426, 2.16821198],
        [0.0, 0.0, 2.81166073, 0.00167067353, -6.79997428e-07, 1.32881379e-10,
         -1.02767442e-14, -869.811579, 6.6483805],
    ])

O2 = dict(
    name="O2", W=31.998, a=149772.3334866597, b=0.01982709144373723, omega=0.0222,
    ranges=[148.0, 182.34, 200.0, 700.0, 3500.0],
    nasa9=[
        [-1008.7297701747248, 38.39770735944911, 2.905984455257836, 0.004775589822483856,
         -2.042411776311955e-05, 4.147926112664399e-08, -2.4757854194367933e-11,
         -1191.2736858521064, 7.404452100810184],
        [0.0, 0.0, 3.487351092425565, 0.000171511121910552, -4.914758364368369e-07,
         -3.668154124316966e-09, 1.714379649770826e-11, -1044.808865594206, 4.770321126998205],
        [0.0, 0.0, 3.74403921, -0.00279740147, 9.80122558e-06, -1.03259643e-08,
         3.79931247e-12, -1060.69827, 3.82132646],
        [0.0, 0.0, 2.82012408, 0.00248211357, -1.51202094e-06, 4.48556201e-10,
         -4.87305668e-14, -931.350148, 7.94914552],
    ])

IC3H7OH = dict(
    name="IC3H7OH", W=60.096, a=1714219.955013869, b=0.06901149227230957, omega=0.6689,
    ranges=[182.34, 300.0, 1490.0, 3500.0],
    nasa9=[
        [0.0, 0.0, 8.268209412358907, -0.08603907736461355, 0.000757315345210363,
         -2.10122524775172e-06, 2.078637900786288e-09, -34964.21834756644, -3.480543450971361],
        [0.0, 0.0, -1.25951086, 0.0499518902, -3.76786393e-05, 1.49318826e-08,
         -2.3934462e-12, -34344.3869, 31.0096138],
        [0.0, 0.0, 10.2736687, 0.0189903342, -6.50928762e-06, 9.8586399e-10,
         -5.35101895e-14, -37781.2744, -29.2304676],
    ])

# The production gas of the reference's impingement case (cold-pr-148K.yaml:6-25):
# air (N2, O2), N2O and isopropanol in one Peng-Robinson phase.
AIR_N2O_IPA = (N2, O2, N2O, IC3H7OH)

# Flash controls of the N2O case (cold-pr-148K-config.yaml:1-19).
N2O_FLASH = dict(liquidTmin=148.0, liquidTc=309.52, Tmin=148.0, Tmax=3500.0,
                 pmin=1000.0, pmax=5.0e7, vtol=1e-9, etol=1e-9, mutol=1e-7)


def kappa(omega):
    """Peng-Robinson kappa(omega), both branches (reactiveDevicePRExport.h:89-92)."""
    if omega <= 0.491:
        return 0.37464 + 1.54226 * omega - 0.26992 * omega * omega
    return 0.374642 + 1.487503 * omega - 0.164423 * omega * omega + 0.016666 * omega ** 3


def critical_point(sp):
    """(Tc [K], pc [Pa]) implied by the PR a and b of one species."""
    tc = sp["a"] * OMEGA_B / (sp["b"] * OMEGA_A * GAS_CONSTANT)
    return tc, OMEGA_B * GAS_CONSTANT * tc / sp["b"]


def _fill_species(dst, sp):
    dst.molecularWeight = sp["W"]
    dst.a = sp["a"]
    dst.b = sp["b"]
    dst.kappa = kappa(sp["omega"])
    dst.regionCount = len(sp["nasa9"])
    for r, coeffs in enumerate(sp["nasa9"]):
        reg = dst.regions[r]
        reg.minimumTemperature = sp["ranges"][r]
        reg.maximumTemperature = sp["ranges"][r + 1]
        reg.polynomial = 9
        for j, a in enumerate(coeffs):
            reg.coefficient[j] = a


def _fill_table(table, species):
    table.ns = len(species)
    table.refPressure = ONE_ATM
    for k, sp in enumerate(species):
        _fill_species(table.species[k], sp)
    for i, si in enumerate(species):
        for j, sj in enumerate(species):
            table.aBinary[i][j] = math.sqrt(si["a"] * sj["a"]) if i != j else si["a"]


def pure_model(sp=N2O, controls=N2O_FLASH, analytic_jacobian=1, scalar_recovery=1,
               boundary_recovery=0, stable_gas_prune=0, enforce_bounds=1):
    """HEM model image for one condensable species with its own pure liquid.

    Gas table and liquid table are the same one-species PR table (ns=1, nl=1,
    condensable[0]=0), which is how the reference exports a pure fluid.
    """
    m = HemModel()
    _fill_table(m.phase[0], [sp])
    _fill_table(m.phase[1], [sp])
    m.ns, m.nl = 1, 1
    m.condensable[0] = 0
    m.boundaryRecovery = boundary_recovery
    m.scalarRecovery = scalar_recovery
    m.analyticJacobian = analytic_jacobian
    m.stableGasPrune = stable_gas_prune
    m.weights[0] = sp["W"]
    m.liquidTmin[0] = controls["liquidTmin"]
    m.liquidTc[0] = controls["liquidTc"]
    for key in ("Tmin", "Tmax", "pmin", "pmax", "vtol", "etol", "mutol"):
        setattr(m, key, controls[key])
    m.enforceSpeciesTemperatureBounds = enforce_bounds
    return m


def mixture_model(species=AIR_N2O_IPA):
    """A HEM model image whose gas table (phase 0) is the Peng-Robinson mixture of
    `species`; used to evaluate mixture properties through the image's table."""
    m = HemModel()
    _fill_table(m.phase[0], list(species))
    m.ns = len(species)
    return m


def production_model(species=AIR_N2O_IPA, condensable="N2O", controls=N2O_FLASH, analytic_jacobian=1,
                     scalar_recovery=1, boundary_recovery=0, enforce_bounds=1):
    """HEM model image of the reference's production configuration
    (cold-pr-148K-config.yaml): the Peng-Robinson gas of `species` and one
    condensed phase, the pure liquid of `condensable` (N2O), with the case's
    bounds and tolerances."""
    m = mixture_model(species)
    k = [sp["name"] for sp in species].index(condensable)
    _fill_table(m.phase[1], [species[k]])
    m.nl = 1
    m.condensable[0] = k
    m.boundaryRecovery = boundary_recovery
    m.scalarRecovery = scalar_recovery
    m.analyticJacobian = analytic_jacobian
    for i, sp in enumerate(species):
        m.weights[i] = sp["W"]
    m.liquidTmin[0] = controls["liquidTmin"]
    m.liquidTc[0] = controls["liquidTc"]
    for key in ("Tmin", "Tmax", "pmin", "pmax", "vtol", "etol", "mutol"):
        setattr(m, key, controls[key])
    m.enforceSpeciesTemperatureBounds = enforce_bounds
    return m


def two_liquid_model(species=AIR_N2O_IPA, condensables=("N2O", "IC3H7OH"), controls=N2O_FLASH, scalar_recovery=1,
                     boundary_recovery=1, stable_gas_prune=0, enforce_bounds=1):
    """HEM model image with two condensed phases: the Peng-Robinson gas of
    `species` and the pure liquids of `condensables` (N2O and isopropanol, the
    configuration the reference's captured recovery inputs were taken with),
    the boundary recovery on, and the Newton Jacobian by finite differences
    (analyticJacobian 0). N2O's liquid range is the case's; isopropanol's runs
    from the start of its NASA data to its Peng-Robinson critical temperature."""
    m = mixture_model(species)
    names = [sp["name"] for sp in species]
    for i, name in enumerate(condensables):
        k = names.index(name)
        _fill_table(m.phase[i + 1], [species[k]])
        m.condensable[i] = k
        if name == "N2O":
            m.liquidTmin[i], m.liquidTc[i] = controls["liquidTmin"], controls["liquidTc"]
        else:
            m.liquidTmin[i], m.liquidTc[i] = species[k]["ranges"][0], critical_point(species[k])[0]
    m.nl = len(condensables)
    m.boundaryRecovery = boundary_recovery
    m.scalarRecovery = scalar_recovery
    m.analyticJacobian = 0
    m.stableGasPrune = stable_gas_prune
    for i, sp in enumerate(species):
        m.weights[i] = sp["W"]
    for key in ("Tmin", "Tmax", "pmin", "pmax", "vtol", "etol", "mutol"):
        setattr(m, key, controls[key])
    m.enforceSpeciesTemperatureBounds = enforce_bounds
    return m


def model_bytes(model):
    return bytes(C.string_at(C.addressof(model), C.sizeof(model)))


def gas_table(species=(N2O, N2)):
    """ReactiveB200Table image (the HEM model image's gas-table layout) of an
    ideal-gas mixture; the ideal-gas closure reads the NASA regions and W."""
    from ._abi import Table
    t = Table()
    _fill_table(t, list(species))
    return bytes(C.string_at(C.addressof(t), C.sizeof(t)))


def nasa_region(sp, T):
    """Index of the NASA region of species sp that holds temperature T (the
    device rule: a NASA9 region starts at its lower bound inclusive)."""
    r = 0
    for j in range(1, len(sp["nasa9"])):
        if T >= sp["ranges"][j]:
            r = j
    return r


def ideal_energy(sp, T, xp=np):
    """Ideal-gas e = h - R T per mass [J/kg] of species sp at temperature T
    (array of one NASA region, or a torch tensor with xp=torch)."""
    r = GAS_CONSTANT / sp["W"]
    region = nasa_region(sp, float(xp.max(T)) if xp is np else float(T.detach().max()))
    a = sp["nasa9"][region]
    iT = 1 / T
    lT = xp.log(T)
    hRT = (-a[0] * iT * iT + lT * a[1] * iT + a[2] + .5 * a[3] * T + a[4] * T * T / 3.0
           + .25 * a[5] * T ** 3 + .2 * a[6] * T ** 4 + a[7] * iT)
    return r * T * (hRT - 1)


def ideal_cv(sp, T, xp=np):
    """Ideal-gas cv = cp - R per mass [J/(kg K)] of species sp (one NASA region)."""
    r = GAS_CONSTANT / sp["W"]
    region = nasa_region(sp, float(xp.max(T)) if xp is np else float(T.detach().max()))
    a = sp["nasa9"][region]
    iT = 1 / T
    cpR = a[0] * iT * iT + a[1] * iT + a[2] + a[3] * T + a[4] * T * T + a[5] * T ** 3 + a[6] * T ** 4
    return r * (cpR - 1)
