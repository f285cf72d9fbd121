"""The CUDA engine against the committed golden fixtures (tests/golden):
fields and probe traces bit for bit, energies to 1e-10, in both kernel
families."""
import pytest

from scenarios import run_engine
from test_golden import MANIFEST, load, scenario
from test_gpu_parity import assert_parity

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernels", ("register", "staged"))
@pytest.mark.parametrize("name", sorted(MANIFEST))
def test_engine_matches_fixture(name, kernels):
    g = load(name)
    ref = {"fields": g["fields"], "timestep": int(g["timestep"]),
           "traces": g.get("traces"), "energy": [tuple(row) for row in g["energy"]]}
    assert_parity(run_engine(scenario(name), kernels=kernels), ref)
