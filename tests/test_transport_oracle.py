"""CPU: pins the transport oracle (oracle/transport_oracle.c) against the
reference's own CPU transport build (oracle/_ref, backend 0) by running the
reference's RHS / CFL / RK-stage / residency contract on the reference library
and checking every number against the oracle."""
import pytest

from oracle import oracle
import transport_cases as T

pytestmark = pytest.mark.filterwarnings("ignore")


@pytest.fixture(scope="module")
def ref():
    return T.bind(oracle.ref_transport_lib())


@pytest.mark.parametrize("spec", T.CASES, ids=lambda s: "-".join(map(str, s)))
def test_oracle_matches_reference_cpu(ref, spec):
    case = T.case_from_tuple(spec)
    summary = T.contract_walk(ref, 0, case, oracle)
    assert summary["rhs_error"] <= T.RHS_TOL


@pytest.mark.parametrize("nc", [65535, 65536, 65537])
def test_reference_large_cfl(ref, nc):
    T.large_cfl_walk(ref, 0, nc)
