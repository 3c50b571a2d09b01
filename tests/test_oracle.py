"""Pin the CPU f64 oracle against the reference's own golden vectors.

Each test mirrors a reference test (named in its docstring) and uses the values
tests/golden/make_golden.py read out of that test's data.  The oracle is the
checker every GPU parity test trusts, so it is checked first.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import golden, golden_nonbonded_system


def test_threefry_known_answers(oracle):
    """test/random.test.ts:39-66 -- Random123 kat_vectors at 13/20/32 rounds."""
    import ctypes as C

    cases = golden("random_kat")["cases"]
    assert len(cases) == 9
    for case in cases:
        out = (C.c_uint32 * 2)()
        c0, c1, k0, k1 = case["input"]
        oracle.lib().orc_threefry2x32(c0, c1, k0, k1, case["rounds"], out)
        assert [out[0], out[1]] == case["output"], case


def test_open_unit_interval_never_reaches_the_ends(oracle):
    """random.ts:102 -- midpoint of 2^23 buckets, strictly inside (0, 1)."""
    lo = oracle.lib().orc_open_unit_interval(0)
    hi = oracle.lib().orc_open_unit_interval(0xFFFFFFFF)
    assert 0 < lo < 1e-6 and 1 - 1e-6 < hi < 1


def test_thermostat_normals_are_standard(oracle):
    draws = np.array([oracle.lib().orc_thermostat_normal(7, s, i, a)
                      for s in range(20) for i in range(200) for a in range(3)])
    assert abs(draws.mean()) < 0.05
    assert abs(draws.std() - 1) < 0.05


def test_erf_matches_mpmath(oracle):
    """test/erf.test.ts:5-45."""
    for x, erf, erfc in golden("erf")["rows"]:
        assert abs(oracle.lib().orc_erf(x) - erf) < 1e-14
        assert abs(oracle.lib().orc_erf(-x) + erf) < 1e-14
        assert abs((oracle.lib().orc_erfc(x) - erfc) / erfc) < 1e-13
        assert abs((oracle.lib().orc_erfc(-x) - (2 - erfc)) / (2 - erfc)) < 1e-13


def test_fixed_words(oracle):
    """test/fixed-point.test.ts:58-62 exact layouts, plus sign symmetry."""
    import ctypes as C

    for case in golden("fixed_words")["cases"]:
        lo, hi = C.c_uint32(), C.c_int32()
        assert oracle.lib().orc_fixed_words(case["value"], C.byref(lo), C.byref(hi)) == 0
        assert (lo.value, hi.value) == (case["lo"], case["hi"])
    rng = np.random.default_rng(3)
    for v in (rng.uniform(-1, 1, 2000) * 10.0 ** rng.uniform(-4, 4, 2000)).astype(np.float32):
        lo, hi = C.c_uint32(), C.c_int32()
        oracle.lib().orc_fixed_words(float(v), C.byref(lo), C.byref(hi))
        fixed = hi.value * 2**32 + lo.value
        lo2, hi2 = C.c_uint32(), C.c_int32()
        oracle.lib().orc_fixed_words(float(-v), C.byref(lo2), C.byref(hi2))
        assert fixed == -(hi2.value * 2**32 + lo2.value)
        assert abs(fixed / 2**32 - float(v)) <= 2.0**-33
    lo, hi = C.c_uint32(), C.c_int32()
    assert oracle.lib().orc_fixed_words(2.0**31, C.byref(lo), C.byref(hi)) == 7  # MDB_ERR_RANGE
    assert oracle.lib().orc_fixed_words(float("nan"), C.byref(lo), C.byref(hi)) == 7


def test_alpha_and_grid_rules(oracle):
    """units.test / pme-reference.test.ts:142 -- alpha 2.628... and the smooth grid."""
    lib = oracle.lib()
    assert abs(lib.orc_ewald_alpha(1.0, 5e-4) - 2.628260884878466) < 1e-14
    g = golden("nonbonded")
    assert abs(lib.orc_ewald_alpha(g["cutoff"], g["ewald_tolerance"]) - g["PME"]["alpha_per_nm"]) < 1e-12
    assert lib.orc_pme_minimum_grid(g["PME"]["alpha_per_nm"], 2.4, 5e-4) == g["PME"]["grid"][0]
    assert lib.orc_smooth_fft_size(53) == 54 and lib.orc_smooth_fft_size(25) == 25
    assert lib.orc_smooth_fft_size(11) == 12


def test_direct_group_term_by_term(oracle):
    """test/nonbonded-reference.test.ts:68-87 -- OpenMM's direct group."""
    system, state, g = golden_nonbonded_system()
    e, _ = oracle.potential(system, state.positions, naive=True, forces=False)
    d = g["decomposition"]
    assert abs(e["direct_coulomb"] - d["direct_coulomb"]) < 1e-9
    assert abs(e["direct_lj"] - d["direct_lj"]) < 1e-9
    assert abs(e["exclusion_correction"] - d["exclusion_correction"]) < 1e-8
    assert abs(e["exceptions"] - d["exception_energy"]) < 1e-8
    assert abs(e["direct_group"] - g["PME"]["direct_group"]) < 1e-6
    assert abs(e["self_energy"] - d["self_energy"]) < 1e-8


def test_dispersion_correction_against_openmm(oracle):
    """test/nonbonded-reference.test.ts:95 -- -0.020466041 kJ/mol."""
    system, state, g = golden_nonbonded_system()
    e, _ = oracle.potential(system, state.positions, naive=True, forces=False)
    assert abs(e["dispersion"] - g["dispersion_openmm"]) < 1e-9


def test_reciprocal_group_against_openmm(oracle):
    """test/pme-reference.test.ts:118-140 -- the 22^3 (non-smooth) mesh, 1e-4 abs."""
    system, state, g = golden_nonbonded_system()
    e, _ = oracle.potential(system, state.positions, grid=g["PME"]["grid"], forces=False)
    assert abs(e["reciprocal_group"] - g["PME"]["reciprocal_group"]) < 1e-4
    assert abs(e["potential"] - g["PME"]["total"]) < 1e-4


def test_pme_forces_against_openmm(oracle):
    """The PME per-atom forces of nonbonded-facts.json."""
    system, state, g = golden_nonbonded_system()
    _, f = oracle.potential(system, state.positions, grid=g["PME"]["grid"])
    want = np.array(g["PME"]["forces"])
    rel = np.sqrt(((f - want) ** 2).sum() / (want**2).sum())
    assert rel < 1e-5, rel


def test_forces_match_numeric_derivative(oracle):
    """test/nonbonded-reference.test.ts:121-146, on the whole potential."""
    system, state, g = golden_nonbonded_system()
    _, f = oracle.potential(system, state.positions, grid=(24, 24, 24))
    pos = state.positions.copy()
    h = 1e-6
    for i in range(pos.shape[0]):
        for a in range(3):
            orig = pos[i, a]
            pos[i, a] = orig + h
            ep, _ = oracle.potential(system, pos, grid=(24, 24, 24), forces=False)
            pos[i, a] = orig - h
            em, _ = oracle.potential(system, pos, grid=(24, 24, 24), forces=False)
            pos[i, a] = orig
            num = -(ep["potential"] - em["potential"]) / (2 * h)
            mag = max(abs(num), abs(f[i, a]), 1.0)
            assert abs(f[i, a] - num) / mag < 1e-6, (i, a, f[i, a], num)


def test_exact_ewald_against_openmm(oracle):
    """The Ewald facts: exact k-space sum + the same direct/self terms."""
    system, state, g = golden_nonbonded_system()
    alpha = g["Ewald"]["alpha_per_nm"]
    erec, _ = oracle.ewald_reciprocal(system, state.positions, alpha, 12)
    d = g["decomposition"]
    assert abs(erec - d["reciprocal_brute_force"]) < 1e-6 * abs(d["reciprocal_brute_force"])


def test_triclinic_minimum_image_against_openmm(oracle):
    """test/triclinic.test.ts -- OpenMM's separations for cube/dodeca/octa."""
    import ctypes as C

    lib = oracle.lib()
    dp = C.POINTER(C.c_double)
    for case in golden("triclinic")["cases"]:
        box = np.ascontiguousarray(np.array(case["reduced_vectors"], dtype=np.float64).reshape(9))
        cutoff = case["cutoff_nm"]
        checked = 0
        for pair in case["pairs"]:
            d = np.ascontiguousarray(np.array(pair["separation"], dtype=np.float64))
            out = np.zeros(3)
            lib.orc_minimum_image(box.ctypes.data_as(dp), d.ctypes.data_as(dp), out.ctypes.data_as(dp))
            search = np.zeros(3)
            lib.orc_nearest_image_by_search(box.ctypes.data_as(dp), d.ctypes.data_as(dp),
                                            search.ctypes.data_as(dp))
            assert abs(np.linalg.norm(search) - pair["brute"]) < 1e-9
            if pair["brute"] < cutoff:
                assert abs(np.linalg.norm(out) - pair["openmm"]) < 1e-9
                checked += 1
        assert checked > 0


def test_reduce_box_is_identity_on_reduced_shapes(oracle):
    import ctypes as C

    dp = C.POINTER(C.c_double)
    for case in golden("triclinic")["cases"]:
        box = np.ascontiguousarray(np.array(case["reduced_vectors"], dtype=np.float64).reshape(9))
        out = np.zeros(9)
        oracle.lib().orc_reduce_box(box.ctypes.data_as(dp), out.ctypes.data_as(dp))
        assert np.array_equal(out, box)


def test_bspline_partition_of_unity_and_moduli(oracle):
    """test/pme-reference.test.ts:16-60 -- weights sum to one, first moment."""
    import ctypes as C

    dp = C.POINTER(C.c_double)
    for w in np.linspace(0, 0.999, 37):
        wt, dv = np.zeros(5), np.zeros(5)
        oracle.lib().orc_bspline(float(w), wt.ctypes.data_as(dp), dv.ctypes.data_as(dp))
        assert abs(wt.sum() - 1) < 1e-14
        assert abs(dv.sum()) < 1e-13
    mod = np.zeros(30)
    oracle.lib().orc_bspline_moduli(30, mod.ctypes.data_as(dp))
    assert np.all(mod > 0) and abs(mod[0] - 1) < 1e-12


def test_cutoff_shell_lists_pairs_at_the_cutoff(oracle):
    """Pairs within eps of the cutoff, with the force each would add if inside
    (erfc-Coulomb plus LJ at the pair's own distance); pairs farther away and
    excluded pairs are not listed."""
    from mdb200.system import Nonbonded, System

    cut, alpha = 1.0, oracle.lib().orc_ewald_alpha(1.0, 5e-4)
    d = [cut - 5e-8, cut + 5e-8, cut - 1e-3]
    pos = np.array([[1, 1, 1], [1 + d[0], 1, 1], [1, 3.5, 1], [1, 3.5 + d[1], 1], [3, 5, 5], [3 + d[2], 5, 5],
                    [6, 1, 1], [6, 1 + cut - 1e-8, 1]], dtype=np.float64)
    q = np.array([0.5, -0.7, 0.4, 0.4, 1.0, -1.0, 0.3, 0.3])
    system = System(masses=np.ones(8), box=np.eye(3) * 9.0,
                    nonbonded=Nonbonded(cutoff=cut, ewald_tolerance=5e-4, charge=q, sigma=np.full(8, 0.3),
                                        epsilon=np.full(8, 0.5),
                                        exception_p1=np.array([6], np.int32), exception_p2=np.array([7], np.int32),
                                        exception_charge_prod=np.zeros(1), exception_sigma=np.full(1, 0.3),
                                        exception_epsilon=np.zeros(1)))
    first, second, force, inside = oracle.cutoff_shell(system, pos, eps=2e-7)
    assert sorted(zip(first.tolist(), second.tolist())) == [(0, 1), (2, 3)]
    for a, b, f, ins in zip(first, second, force, inside):
        r = float(np.linalg.norm(pos[b] - pos[a]))
        assert ins == (r < cut)
        qq = 138.935458 * q[a] * q[b]
        s6 = (0.3 / r) ** 6
        dedr = qq * (-math.erfc(alpha * r) / r**2 - alpha * 2 / math.sqrt(math.pi) * math.exp(-(alpha * r) ** 2) / r)
        dedr += 4 * 0.5 / r * (6 * s6 - 12 * s6 * s6)
        np.testing.assert_allclose(f, dedr / r * (pos[b] - pos[a]), rtol=1e-6)
