"""The CPU oracle: the C restatement against the reference and its fixtures.

The fixtures in tests/golden/ come from running the reference's own step
(tests/golden/gen_golden.py); these tests pin the restatement to them. Where
the reference build (oracle/_ref) is present, the restatement is also checked
routine by routine against it directly.
"""
import numpy as np
import pytest

from conftest import golden, kat_state, rel_l2

ROUTINES = ["pzeta_pt", "pth_pt", "pqv_pt", "pqc_pt", "pqr_pt", "BoundaryProcess2D_all",
            "pubarTop_pt", "cal_w", "cal_u", "autoconversion", "accretion", "evaporation",
            "condensation", "NVP_qvp", "NVP_qcp", "NVP_qrp", "updateMean", "RKM_RKH",
            "Nudge_theta", "Nudge_zeta", "nextTimeStep"]
ELLIPTIC = {"cal_w": 1e-12, "cal_u": 1e-12}   # exact solves vs iterative (round-off)


def test_initial_state_is_pinned():
    """The synthetic warm bubble reproduces the fixture bit for bit."""
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble()
    z = golden("config1_init.npz")
    for k, v in st.fields.items():
        assert np.array_equal(v, z[f"f_{k}"]), k
    for k, v in st.prof.items():
        assert np.array_equal(v, z[f"p_{k}"]), k


@pytest.mark.parametrize("routine", ROUTINES)
def test_port_routine_matches_reference_fixture(routine, port_lib):
    st, z = kat_state()
    m = port_lib.PortModel(st.grid)
    m.load(st)
    m.call(routine)
    d = m.dump()
    tol = ELLIPTIC.get(routine, 0.0)
    checked = 0
    for key in z.files:
        if not key.startswith(routine + "__"):
            continue
        name = key.split("__", 1)[1]
        ref = z[key]
        if name.startswith("h_"):
            got = d.hist[name[2:]]
        elif name.startswith("p_"):
            got = d.prof[name[2:]]
        elif name == "precip":
            got = d.precip
        elif name == "ubarTopp":
            got = np.array(d.scalars["ubarTopp"])
        elif name == "dubar":
            got = d.scalars["dubarTop_advect"]
        else:
            got = d.fields[name]
        if tol == 0.0:
            assert np.array_equal(got, ref, equal_nan=True), f"{routine}: {name} not bit-exact"
        else:
            assert rel_l2(got, ref) <= tol, f"{routine}: {name} {rel_l2(got, ref):.2e}"
        checked += 1
    assert checked >= 2


def test_port_steps_match_reference_fixtures(port_lib):
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble()
    m = port_lib.PortModel(st.grid)
    m.load(st)
    for nstep, tol in ((1, 1e-11), (10, 1e-9)):
        while m.step < nstep:
            m.one_step()
        z = golden(f"config1_step{nstep}.npz")
        d = m.dump()
        for f in ("zeta", "th", "qv", "qc", "qr", "u", "w"):
            assert rel_l2(d.fields[f], z[f]) <= tol, (nstep, f, rel_l2(d.fields[f], z[f]))


def test_port_poisson_manufactured_solution(port_lib):
    """Exact solve of A x = b for x = exp(sin(i + k)) (the reference's
    POISSONTEST construction) and the reference's own matrix-vector product."""
    from vvm_b200.initial_state import warm_bubble
    z = golden("poisson_kat.npz")
    st = warm_bubble(int(z["NX"]), int(z["NZ"]))
    assert np.array_equal(st.prof["rhou"], z["rhou"])
    m = port_lib.PortModel(st.grid)
    m.load(st)
    assert rel_l2(m.apply_A(z["x_ans"]), z["b"]) <= 1e-15
    x = m.solve_A(z["b"])
    assert rel_l2(x, z["x_ans"]) <= 1e-12
    assert rel_l2(z["x_ref"], z["x_ans"]) <= 1e-10   # the reference's BiCGSTAB
    assert float(z["true_relres"]) <= 1e-12


def test_port_600_steps_domain_means(port_lib):
    """Domain means of 600 restated steps against the reference's run."""
    from vvm_b200.initial_state import warm_bubble
    from tests_helpers import domain_means
    st = warm_bubble()
    m = port_lib.PortModel(st.grid)
    m.load(st)
    for _ in range(600):
        m.one_step()
    z = golden("config1_600.npz")
    got = domain_means(m.dump())
    ref = z["means"][-1]
    assert abs(got[0] - ref[0]) / abs(ref[0]) <= 1e-12        # th
    for j in (1, 2, 3, 4):                                     # qc, qr, rain, KE
        assert abs(got[j] - ref[j]) <= 1e-6 * max(abs(ref[j]), 1e-30), (j, got[j], ref[j])


@pytest.mark.skipif("not __import__('oracle.models', fromlist=['x']).ref_available()")
class TestAgainstReferenceBuild:
    """Direct comparisons with the reference's own step (oracle/_ref)."""

    def test_one_step_replica_equals_time_marching(self):
        from oracle.models import RefModel
        from vvm_b200.initial_state import warm_bubble
        st = warm_bubble(64, 32)
        a = RefModel(st.grid)
        a.load(st)
        for _ in range(5):
            a.one_step()
        b = RefModel(st.grid)
        b.load(st)
        b.time_marching(5)
        da, db = a.dump(), b.dump()
        for f in da.fields:
            assert np.array_equal(da.fields[f], db.fields[f]), f

    def test_reference_reproduces_fixtures(self):
        from oracle.models import RefModel
        from vvm_b200.initial_state import warm_bubble
        st = warm_bubble()
        m = RefModel(st.grid)
        m.load(st)
        m.one_step()
        z = golden("config1_step1.npz")
        d = m.dump()
        for f in ("zeta", "th", "qv", "qc", "qr", "u", "w"):
            assert np.array_equal(d.fields[f], z[f]), f

    @pytest.mark.parametrize("seed", [1, 2])
    def test_port_equals_reference_per_routine(self, seed, port_lib):
        from oracle.models import RefModel
        from vvm_b200.initial_state import random_state
        st = random_state(24, 20, seed=seed)
        for n in ("zetap", "thp", "qvp", "qcp", "qrp"):
            st.fields[n] = st.fields[n[:-1]] * 0.99
        for r in ROUTINES:
            a = RefModel(st.grid)
            a.load(st)
            a.call(r)
            b = port_lib.PortModel(st.grid)
            b.load(st)
            b.call(r)
            da, db = a.dump(), b.dump()
            tol = ELLIPTIC.get(r, 0.0)
            for f in da.fields:
                if tol:
                    assert rel_l2(db.fields[f], da.fields[f]) <= tol, (r, f)
                else:
                    assert np.array_equal(db.fields[f], da.fields[f], equal_nan=True), (r, f)


def _halo_state():
    st, _ = kat_state()
    z = golden("halo_kat.npz")
    for n in ("zetap", "thp", "w", "u", "qvp", "qcp", "qrp"):
        st.fields[n] = z[f"in_{n}"].copy()
    return st, z


def test_port_halo_all_rewrites_scrambled_ghosts(port_lib):
    """BoundaryProcess2D_all on a state whose ghost cells hold noise: every
    ghost is rewritten from the interior exactly as the reference does."""
    st, z = _halo_state()
    m = port_lib.PortModel(st.grid)
    m.load(st)
    m.call("BoundaryProcess2D_all")
    for n in ("zetap", "thp", "w", "u", "qvp", "qcp", "qrp"):
        assert not np.array_equal(z[f"in_{n}"], z[f"out_{n}"]), n   # the call changed something
        assert np.array_equal(m.field(n), z[f"out_{n}"]), n


class TestStreamfunction:
    """The streamfunction formulation (STREAMFUNCTION): the restatement's
    exact solve against the reference built with it (fixture
    stream_kat.npz; POISSONPARAM = 0)."""

    def test_port_calpsiuw_matches_reference_fixture(self, port_lib):
        st, _ = kat_state()
        z = golden("stream_kat.npz")
        m = port_lib.PortModel(st.grid)
        m.load(st)
        m.call("calpsiuw")
        for n in ("psi", "u", "w"):
            assert rel_l2(m.field(n), z[f"calpsiuw__{n}"]) <= 1e-12, (n, rel_l2(m.field(n), z[f"calpsiuw__{n}"]))

    def test_port_psi_solution_meets_the_reference_matrix(self, port_lib):
        """psi solves the reference's psi matrix (src/PoissonSolver.cpp:726-756)
        to round-off: ||b - A psi|| / ||b|| with b = zetap dx^2."""
        st, _ = kat_state()
        m = port_lib.PortModel(st.grid)
        m.load(st)
        m.call("calpsiuw")
        x = m.field("psi")[1:-1, 2:-1].T.reshape(-1)
        b = (st.fields["zetap"][1:-1, 2:-1] * st.grid.dx ** 2).T.reshape(-1)
        assert np.linalg.norm(b - m.apply_psi(x)) / np.linalg.norm(b) <= 1e-13

    @pytest.mark.parametrize("steps", [1, 10])
    def test_port_stream_steps_match_reference_fixture(self, steps, port_lib):
        from vvm_b200.initial_state import warm_bubble
        st = warm_bubble(64, 32)
        z = golden("stream_kat.npz")
        m = port_lib.PortModel(st.grid)
        m.load(st)
        m.set_streamfunction(True)
        for _ in range(steps):
            m.one_step()
        for n in ("zeta", "th", "qv", "u", "w", "psi"):
            bound = 1e-13 if n in ("th", "qv") else 1e-10
            e = rel_l2(m.field(n), z[f"step{steps}__{n}"])
            assert e <= bound, (n, e)

    def test_reference_stream_build_reproduces_fixture(self):
        from oracle.models import RefStreamModel, ref_stream_available
        if not ref_stream_available():
            pytest.skip("oracle/_ref/libvvmref_stream.so is not built")
        st, _ = kat_state()
        z = golden("stream_kat.npz")
        m = RefStreamModel(st.grid)
        m.load(st)
        m.call("calpsiuw")
        assert np.array_equal(m.psi(), z["calpsiuw__psi"])
        assert np.array_equal(m.field("w"), z["calpsiuw__w"])


class TestThreadedBaseline:
    """The race-free multi-core CPU baseline (oracle/_build/libvvmoracle_mt.so):
    the restatement with OpenMP loops and FFT-based cal_w equals the serial
    restatement to round-off, with more than one thread."""

    @pytest.fixture(scope="class")
    def models(self):
        from oracle import models
        if not models.port_mt_available():
            import subprocess
            from conftest import REPO
            subprocess.run(["make", "-s", "-C", str(REPO / "oracle")], check=True)
        return models

    @pytest.mark.parametrize("NX,NZ", [(128, 64), (48, 20)])   # FFT path, DFT path
    def test_threaded_steps_equal_serial(self, models, NX, NZ):
        from vvm_b200.initial_state import random_state
        st = random_state(NX, NZ, seed=4)
        a = models.PortModel(st.grid)
        a.load(st)
        b = models.PortMTModel(st.grid)
        b.load(st)
        assert b.threads() >= 1
        for _ in range(3):
            a.one_step()
            b.one_step()
        for n in ("zeta", "th", "qv", "qc", "qr", "u", "w"):
            assert rel_l2(b.field(n), a.field(n)) <= 1e-12, n

    def test_fft_cal_w_meets_the_reference_matrix(self, models):
        from vvm_b200.initial_state import warm_bubble
        st = warm_bubble(256, 32)
        m = models.PortMTModel(st.grid)
        m.load(st)
        rng = np.random.default_rng(3)
        b = rng.standard_normal(st.grid.NX * (st.grid.NZ - 1))
        x = m.solve_A(b)
        assert np.linalg.norm(b - m.apply_A(x)) / np.linalg.norm(b) <= 1e-13
