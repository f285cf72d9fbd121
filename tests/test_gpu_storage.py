"""2-byte field storage (half / bfloat16, float arithmetic): bit-exact against
the numpy restatement of the same storage rounding, and accurate to a stated
bound against the FP64 oracle; conversions, energies, refusals and a port
sweep.

Every store rounds to 11 (half) or 8 (bfloat16) significant bits, so the
error against FP64 grows with the step count and with how much a field's
small changes sit on a large value: a source with a DC part (a Gaussian
pulse without a carrier) leaves a static charge whose field swallows the
late-time increments of the fields around it in half precision.  The
accuracy tests therefore use a modulated Gaussian; the bounds are about
twice the errors of the numpy restatement (600 steps, 64^3: half 2.0e-2,
bfloat16 1.7e-1)."""
import numpy as np
import pytest

import openems_b200 as oe
from conftest import rel_l2
from oracle.numpy_ref import run_stored
from scenarios import Scenario, make_operator, run_engine, run_oracle

pytestmark = pytest.mark.gpu

BOUND = {"f16": 4e-2, "bf16": 3.5e-1}
CELLS = [(16, 16, 16), (48, 16, 32), (32, 48, 16), (40, 40, 48)]


def modulated_cube(n=64, steps=600, cpml=None):
    c = n // 2
    return Scenario(f"modulated_{n}", (n, n, n), 1e-3,
                    excitations=[oe.Excitation.gaussian_modulated(10e9, 0.5, 2, (c, c, c))], num_steps=steps,
                    sample_interval=100, track_peak=True, cpml=cpml,
                    probes=[(2, p) for p in CELLS if max(p) < n] + [(4, p) for p in CELLS if max(p) < n])


@pytest.mark.parametrize("compressed", [False, True])
@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_bit_exact_against_storage_restatement(storage, compressed):
    """Lossy dielectric, PEC block, a soft and a hard source: the engine's
    2-byte fields equal the numpy restatement bit for bit (same float32
    operations, same rounding on every store)."""
    sc = Scenario("storage_small", (20, 24, 28), 1e-3,
                  materials=[(4.0, 1.0, 0.02, 0.0, (6, 14, 5, 19, 7, 21))], pec=[(9, 11, 2, 22, 3, 5)],
                  excitations=[oe.Excitation.gaussian_modulated(10e9, 0.5, 2, (10, 12, 14)),
                               oe.Excitation.gaussian_modulated(15e9, 0.5, 0, (12, 8, 20)).hard_source()],
                  num_steps=150)
    got = run_engine(sc, compressed=compressed, autotune=False, kernels="register", storage=storage)
    op = make_operator(sc)
    dt = op.timestep()
    exc = [(x.position, x.direction, x.soft_source, x.sample(0, sc.num_steps, dt)) for x in sc.excitations]
    want = run_stored(op.coefficients(), np.zeros((6,) + sc.dims, np.float32), sc.num_steps, exc, store=storage)
    assert got["timestep"] == sc.num_steps
    assert np.abs(want).max() > 0
    assert np.array_equal(got["fields"], want), np.abs(got["fields"] - want).max()


@pytest.mark.parametrize("compressed", [False, True])
@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_pec_cube_against_fp64_oracle(storage, compressed):
    sc = modulated_cube()
    ref = run_oracle(sc, precision=64, threads=8)
    got = run_engine(sc, compressed=compressed, autotune=False, kernels="register", storage=storage)
    e, h = rel_l2(got["fields"][:3], ref["fields"][:3]), rel_l2(got["fields"][3:], ref["fields"][3:])
    tr = rel_l2(got["traces"], ref["traces"])
    print(f"{storage} compressed={compressed}: E {e:.2e} H {h:.2e} probes {tr:.2e}")
    assert e < BOUND[storage] and h < BOUND[storage] and tr < BOUND[storage]
    assert got["timestep"] == ref["timestep"]
    for (t1, e1, _, _), (t2, e2, _, _) in zip(got["energy"], ref["energy"]):
        assert t1 == t2
        assert e1 == pytest.approx(e2, rel=4 * BOUND[storage], abs=1e-300)


@pytest.mark.parametrize("storage", ["f16", "bf16"])
def test_cpml_against_fp64_oracle(storage):
    """With CPML the pulse has left the box after 300 steps: the final fields
    are the small static remainder of the source's DC part (H almost zero),
    whose relative error in 2-byte storage is larger than that of the pulse.
    The run is assessed by the Ez / Hy probe traces over all its steps, the
    final E by twice the bound."""
    sc = modulated_cube(32, 300, oe.CpmlBoundaries.uniform(6))
    sc.probes = [(c, p) for p in [(10, 16, 16), (16, 22, 12), (20, 12, 18)] for c in (2, 4)]
    ref = run_oracle(sc, precision=64, threads=8)
    got = run_engine(sc, autotune=False, kernels="register", storage=storage)
    f32 = run_engine(sc, autotune=False, kernels="register")
    e, tr = rel_l2(got["fields"][:3], ref["fields"][:3]), rel_l2(got["traces"], ref["traces"])
    e32, tr32 = rel_l2(f32["fields"][:3], ref["fields"][:3]), rel_l2(f32["traces"], ref["traces"])
    print(f"{storage} CPML: E {e:.2e} probes {tr:.2e} (f32: E {e32:.2e} probes {tr32:.2e})")
    assert tr < BOUND[storage] and e < 2 * BOUND[storage]


@pytest.mark.parametrize("storage,bits", [("f16", 11), ("bf16", 8)])
def test_write_read_round_trip_and_energy(storage, bits):
    """write_fields rounds to the storage (H after scaling by a power of
    two, so H rounds like E); read_fields gives those values back exactly,
    and the engine's energies are the f64 sums of their squares."""
    dims = (13, 11, 21)
    op = oe.Operator(oe.Grid.uniform(*dims, 1e-3), oe.BoundaryConditions.all_pec())
    eng = oe.Engine(op, storage=storage, kernels="register")
    rng = np.random.default_rng(3)
    f = rng.standard_normal((6,) + dims)
    f = (np.sign(f) * np.maximum(np.abs(f), 0.01)).astype(np.float32)  # clear of half's subnormals
    f[3:] *= 2.7e-3
    eng.write_fields(f[:3], f[3:])
    e, h = eng.read_fields()
    back = np.concatenate([e, h])
    assert np.all(np.abs(back - f) <= 2.0 ** -bits * np.abs(f))
    eng.write_fields(back[:3], back[3:])
    e2, h2 = eng.read_fields()
    assert np.array_equal(np.concatenate([e2, h2]), back)
    ee, he = eng.energy()
    assert ee == pytest.approx(float((back[:3].astype(np.float64) ** 2).sum()), rel=1e-12)
    assert he == pytest.approx(float((back[3:].astype(np.float64) ** 2).sum()), rel=1e-12)


def test_unsupported_combinations_are_refused():
    op = oe.Operator(oe.Grid.uniform(16, 16, 16, 1e-3), oe.BoundaryConditions.all_pec())
    with pytest.raises(oe.ConfigError):
        oe.Engine(op, storage="f16", kernels="staged")
    with pytest.raises(oe.ConfigError):
        oe.Engine(op, storage="f64")
    eng = oe.Engine(op, storage="bf16")
    with pytest.raises(oe.ConfigError):
        eng.add_mur(oe.MurAbcConfig.all(1))
    with pytest.raises(oe.ConfigError):
        eng.add_dispersive(oe.DrudeMaterial(1e10, 1e9), [(3, 3, 3)])


def test_port_sweep_with_half_storage():
    """A patch instance of the port sweep: S11 with half storage against the
    FP32 run (mean |dB| difference over the band, clipped at -30 dB)."""
    from openems_b200 import early_stop as E
    from openems_b200 import workloads as W
    from openems_b200.sweep import Sweep
    spec = W.PatchSpec((40, 33, 28), 2.2, 3, 16, 10, 12, 11, 20, 14, k_ground=8, layers=6)
    freqs = np.linspace(0.5e9, 12e9, 47)
    res = {}
    for st in ("f32", "f16"):
        sw = Sweep(freqs, concurrency=1, storage=st)
        i = sw.add(W.patch_sweep_instance(spec, delta=0.5e-3, decay_db=50.0, max_steps=20000, fmax=12e9))
        sw.run(700)
        res[st] = sw.result(i)
    d = E.s11_db_mean_error(res["f16"]["s11"], res["f32"]["s11"], freqs >= 0.5e9)
    print(f"half-storage sweep: {res['f16']['timesteps']} vs {res['f32']['timesteps']} steps, "
          f"mean S11 difference {d:.3f} dB")
    assert res["f16"]["termination_reason"] == 1
    assert d < 0.5
