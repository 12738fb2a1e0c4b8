"""The physics selection of physics_config.h as run-time options: the
Kieft-Bosch inelastic model and the option bools of every model
(full_penn.h:15-19, kieft/inelastic.h:12-23, kieft/elastic.h:17-22,
boundary_intersect.h:11-19).

CPU only: the library's table preparation and the oracle against the
reference's own templates (oracle/_ref, instantiated with each combination of
option bools): tables bit for bit, single events bit for bit for random
option combinations, and whole driver runs record for record for four
physics presets."""
import numpy as np
import pytest

import nebula_b200 as nb
from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")

PRESETS = {
    "reference": {},
    "kieft": {"inelastic_model": 1},
    "classical_boundary": {"acoustic_phonon_loss": 0, "atomic_recoil_loss": 0, "quantum_transmission": 0,
                           "interface_refraction": 0, "interface_absorption": 1},
    "kieft_plain": {"inelastic_model": 1, "optical_phonon_loss": 0, "instantaneous_momentum": 0,
                    "momentum_conservation": 0},
}


def test_physics_bits_match_library_names():
    # the oracle's bit names are the library's option names
    from nebula_b200 import _capi
    assert set(O.PHYSICS_BITS) | {"inelastic_model"} == set(_capi.PHYSICS_OPTION_NAMES)
    assert O.physics_bits({}) == 0x1DF
    assert O.physics_bits(PRESETS["kieft"]) == 0x101DF
    assert O.physics_bits(PRESETS["classical_boundary"]) == 0x1E1
    assert O.physics_bits(PRESETS["kieft_plain"]) == 0x1001F


def test_physics_options_validated():
    o = nb.physics_options({"interface_refraction": 0})
    assert o.interface_refraction == 0 and o.quantum_transmission == 1
    with pytest.raises(KeyError):
        nb.physics_options({"no_such_option": 1})


@pytest.mark.parametrize("name", ["si", "pmma"])
def test_kieft_tables_library_oracle(inputs, name):
    lib_t = nb.Material.load(inputs[name + "_kieft.nmat"]).tables()
    assert lib_t["models"] == 2
    om = O.Material(inputs[name + "_kieft.nmat"])
    assert om.view.models == 2
    for t in O.KIEFT_TABLE_NAMES + ("el_imfp", "el_icdf"):
        a, sa = lib_t[t]
        b, sb = om.table(t)
        assert a.shape == b.shape, t
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), t
        assert np.array_equal(sa.view(np.uint32), sb.view(np.uint32)), t


@needs_ref
@pytest.mark.parametrize("name", ["si", "pmma"])
def test_kieft_tables_bit_exact_vs_reference(inputs, name):
    """kieft_inelastic::create rewrites its ionisation table in place while
    reading it; the library and the oracle reproduce the result exactly."""
    rm = O.RefMaterial(inputs[name + "_kieft.nmat"])
    lib_t = nb.Material.load(inputs[name + "_kieft.nmat"]).tables()
    for t in O.KIEFT_TABLE_NAMES + ("el_imfp", "el_icdf"):
        a, sa = lib_t[t]
        r, sr = rm.table(t)
        assert np.array_equal(a.reshape(r.shape).view(np.uint32), r.view(np.uint32)), t
        assert np.array_equal(sa.view(np.uint32), sr.view(np.uint32)), t
    assert np.array_equal(nb.Material.load(inputs[name + "_kieft.nmat"]).tables()["constants"].view(np.uint32),
                          rm.constants().view(np.uint32))


def _random_bits(rng, kieft=None):
    b = 0
    for v in O.PHYSICS_BITS.values():
        if rng.random() < 0.5:
            b |= v
    if kieft if kieft is not None else rng.random() < 0.5:
        b |= O.KIEFT_BIT
    return b


@needs_ref
@pytest.mark.parametrize("kind", [1, 2, 3])
def test_events_bit_exact_vs_reference_any_options(inputs, kind):
    """One event per case with random option bools: the oracle and the
    reference templates agree bit for bit (same mt19937 stream)."""
    rg = O.RefGeometry(inputs["grating.tri"])
    og = rg.oracle_geometry()
    rng = np.random.default_rng(100 + kind)
    for model in ("penn", "kieft"):
        suffix = "_kieft.nmat" if model == "kieft" else ".nmat"
        rms = [O.RefMaterial(inputs["si" + suffix]), O.RefMaterial(inputs["pmma" + suffix])]
        oms = [O.Material(inputs["si" + suffix]), O.Material(inputs["pmma" + suffix])]
        for it in range(300):
            bits = _random_bits(rng, kieft=(model == "kieft"))
            E = float(np.exp(rng.uniform(np.log(13), np.log(9000))))
            d = rng.standard_normal(3)
            st = np.array([rng.uniform(-60, 60), rng.uniform(-60, 60), rng.uniform(-50, 30), *d, E], np.float32)
            mat = int(rng.integers(0, 2))
            tri = int(rng.integers(0, len(rg.tri11))) if kind == 3 else -1
            if kind == 3:
                mat = int(rng.choice([0, 1, -123]))
            seed = int(rng.integers(0, 2 ** 32))
            a = O.ref_event(rg, rms, kind, st, mat, seed, tri, phys=bits)
            h = O.lib().orc_rng_mt(seed)
            b = O.event(og, oms, kind, st, mat, h, tri, phys=bits)
            O.lib().orc_rng_free(h)
            ctx = (model, hex(bits), kind, st.tolist(), mat, tri)
            assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32)), ctx
            assert a[1:3] == b[1:3], ctx
            assert (a[3] is None) == (b[3] is None), ctx
            if a[3] is not None:
                assert np.array_equal(a[3].view(np.uint32), b[3].view(np.uint32)), ctx


@needs_ref
@pytest.mark.parametrize("preset", sorted(PRESETS))
def test_driver_records_bit_exact_vs_reference(inputs, preset):
    """Whole CPU-driver runs (grating, a few pixels) for four physics
    presets: identical detected-electron records and event counts."""
    ph = PRESETS[preset]
    bits = O.physics_bits(ph)
    suffix = "_kieft.nmat" if ph.get("inelastic_model") == 1 else ".nmat"
    rg = O.RefGeometry(inputs["grating.tri"])
    og = rg.oracle_geometry()
    rms = [O.RefMaterial(inputs["si" + suffix]), O.RefMaterial(inputs["pmma" + suffix])]
    oms = [O.Material(inputs["si" + suffix]), O.Material(inputs["pmma" + suffix])]
    from nebula_b200.synth import workloads
    w = workloads.grating(pixels=[(100, 120), (140, 30)], per_pixel=40)
    a = O.ref_simulate(rg, rms, w.primaries, 91, phys=bits)
    b = O.simulate(og, oms, w.primaries, 91, phys=bits)
    assert a[1] > 0
    assert a[2] == b[2] and a[1] == b[1]
    assert a[0].tobytes() == b[0].tobytes()


@needs_ref
def test_unknown_preset_is_an_error(inputs):
    rg = O.RefGeometry(inputs["slab.tri"])
    rms = [O.RefMaterial(inputs["si.nmat"])]
    from nebula_b200.synth import primaries
    with pytest.raises(RuntimeError):
        O.ref_simulate(rg, rms, primaries.point_beam(2), 1, phys=0x1)


def test_library_rejects_missing_model_tables(inputs):
    g = nb.Geometry.from_tri_file(inputs["slab.tri"])
    m = nb.Material.load(inputs["si.nmat"])
    from nebula_b200 import _capi
    import ctypes as C
    # a Full-Penn material under the Kieft-Bosch model: rejected before any
    # device work (the check runs first on every machine)
    p = _capi.Params()
    nb.lib().nbl_params_defaults(C.byref(p))
    p.physics = nb.physics_options({"inelastic_model": 1})
    p.capacity = 1024
    h = C.c_void_p()
    arr = (C.c_void_p * 1)(m._h.value if isinstance(m._h, C.c_void_p) else m._h)
    st = nb.lib().nbl_sim_create(g._h, arr, 1, C.byref(p), C.byref(h))
    assert st != 0
    p.physics = nb.physics_options({"interface_refraction": 2})
    st = nb.lib().nbl_sim_create(g._h, arr, 1, C.byref(p), C.byref(h))
    assert st == 1
