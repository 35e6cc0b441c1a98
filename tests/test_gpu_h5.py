"""HDF5 output and restart through the C ABI (ch4_output_h5, ch4_write_pop_h5,
ch4_read_pop_h5) with the reference's layout (src/output_h5.c): the files parse under
the independent spec reader (tests/h5spec.py) and hold exactly the handle's fields and
populations; a handle loaded from pop.h5 is the handle given the same populations with
ch4_set_pop (the reference's resume path, src/initial_conditions.c:606), phases included."""
import numpy as np
import pytest

import h5spec
from lbcases import make_case, pop_items

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

import ch4b200  # noqa: E402
from ch4b200 import abi  # noqa: E402


def started(cfg, state, nsteps):
    sim = ch4b200.Simulation(cfg)
    for k, v in pop_items(state):
        sim.set_pop(k, v)
    sim.initialize()
    sim.step(nsteps)
    return sim


@pytest.mark.parametrize("name", ["rb", "scalar", "hit"])
def test_field_file_holds_the_fields(name, tmp_path):
    _, cfg, state = make_case(name, seed=61)
    with started(cfg, state, 5) as sim:
        sim.output_h5(tmp_path, 5, time_now=5.0, grid=True)
        f = sim.fields()
    got = h5spec.read(tmp_path / "field_5.h5")
    shape = (cfg.NZ, cfg.NY, cfg.NX)
    k, j, i = np.meshgrid(np.arange(cfg.NZ), np.arange(cfg.NY), np.arange(cfg.NX), indexing="ij")
    assert np.array_equal(got["/euler/position_x"], i + 0.5)
    assert np.array_equal(got["/euler/position_y"], j + 0.5)
    assert np.array_equal(got["/euler/position_z"], k + 0.5)
    for a, comp in enumerate("xyz"):
        assert np.array_equal(got["/euler/velocity_" + comp], f["u"][..., a].reshape(shape)), comp
    assert np.array_equal(got["/euler/density"], f["dens"].reshape(shape))
    for flag, key, ds in (("LB_TEMPERATURE", "t", "temperature"), ("LB_SCALAR", "s", "scalar")):
        on = bool(cfg.flags & abi.FLAGS[flag])
        assert ("/euler/" + ds in got) == on, ds
        if on:
            assert np.array_equal(got["/euler/" + ds], f[key].reshape(shape)), ds
    xmf = (tmp_path / "field_5.xmf").read_text()
    assert xmf.startswith('<?xml version="1.0" ?>\n<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>\n')
    assert '<Topology TopologyType="3DSMesh" NumberOfElements="%d %d %d"/>' % shape in xmf
    for ds in [n for n in got if n.startswith("/euler/")]:
        assert "field_5.h5:%s\n" % ds in xmf, ds
    assert xmf.endswith('<Time Value=" 5.000000e+00" />\n</Grid>\n</Domain>\n</Xdmf>\n')


def test_timestamp_and_no_grid(tmp_path):
    _, cfg, state = make_case("rb", seed=62)
    with started(cfg, state, 2) as sim:
        sim.output_h5(tmp_path, 2, time_now=7.9, grid=False, timestamp_real=True)
    got = h5spec.read(tmp_path / "field_7.h5")
    assert "/euler/position_x" not in got and "/euler/velocity_x" in got
    assert '<Topology TopologyType="3DCoRectMesh"' in (tmp_path / "field_7.xmf").read_text()


@pytest.mark.parametrize("name", ["rb", "scalar", "hit"])
def test_pop_file_restart(name, tmp_path):
    _, cfg, state = make_case(name, seed=63)
    path = tmp_path / "pop.h5"
    with started(cfg, state, 6) as a:
        a.write_pop_h5(path)
        pops = {k: a.get_pop(k) for k, _ in pop_items(state)}
        phases = a.get_hit_phases()
    got = h5spec.read(path)
    sets = {"p": "velocity", "g": "temperature", "h": "scalar"}
    for k, arr in pops.items():
        d = got["/population/" + sets[k]]
        assert d.shape == (cfg.NZ, cfg.NY, cfg.NX)
        back = np.stack([d["p%d" % q] for q in range(19)], axis=-1)
        assert np.array_equal(back.reshape(arr.shape), arr), k
    if name == "hit":
        phi = got["/forcing@phi_u"]
        assert got["/forcing@number of modes (nk)"].item() == 6
        assert np.array_equal(np.stack([phi["x"], phi["y"], phi["z"]], 1).ravel(), phases.ravel())
    else:
        assert not any(n.startswith("/forcing") for n in got)
    # resume from the file == the same populations (and phases) given directly
    with ch4b200.Simulation(cfg) as b, ch4b200.Simulation(cfg) as c:
        b.read_pop_h5(path)
        for k, arr in pops.items():
            c.set_pop(k, arr)
        if name == "hit":
            c.set_hit_phases(phases)
            assert np.array_equal(b.get_hit_phases(), phases)
        b.initialize()
        c.initialize()
        b.step(4)
        c.step(4)
        for k in pops:
            assert np.array_equal(b.get_pop(k), c.get_pop(k)), k


def test_read_pop_refuses_a_wrong_lattice(tmp_path):
    _, cfg, state = make_case("rb", seed=64)
    with started(cfg, state, 1) as a:
        a.write_pop_h5(tmp_path / "pop.h5")
    cfg.NX += 1
    cfg.SX += 1
    with ch4b200.Simulation(cfg) as b:
        with pytest.raises(ch4b200.CH4Error):
            b.read_pop_h5(tmp_path / "pop.h5")


def _fields(flags, output_fluid, flags2=0):
    """/lagrange dataset -> ch4_particle field, in output_particles' order."""
    f = [(n, n) for n in ("name", "tau_drag", "x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")]
    grad, am = flags & abi.FLAGS["LAGRANGE_GRADIENT"], flags & abi.FLAGS["LAGRANGE_ADDEDMASS"]
    if grad:  # the fluid and orientation datasets sit inside the gradient block (src/lagrange.c:1783-2014)
        f += [(n, n) for n in ("dx_ux", "dy_ux", "dz_ux", "dx_uy", "dy_uy", "dz_uy", "dx_uz", "dy_uz", "dz_uz")]
        if am:
            f.append(("beta_coeff", "beta_coeff"))
        if output_fluid:
            f += [("ux", "ux"), ("uy", "uy"), ("uz", "uz")]
            if am:
                f += [("Dt_ux", "Dt_ux"), ("Dt_uy", "Dt_uy"), ("Dt_uz", "Dt_uz")]
        if flags & abi.FLAGS["LAGRANGE_ORIENTATION"]:
            f += [(n, n) for n in ("px", "py", "pz", "dt_px", "dt_py", "dt_pz")]
            if flags2 & abi.FLAGS2["LAGRANGE_ORIENTATION_SECONDORIENTATION"]:  # src/lagrange.c:1925-1962
                f += [(n, n) for n in ("nx", "ny", "nz", "dt_nx", "dt_ny", "dt_nz")]
            if flags & abi.FLAGS["LAGRANGE_ORIENTATION_JEFFREY"]:
                f.append(("aspect_ratio", "aspect_ratio"))
                if flags2 & abi.FLAGS2["LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS"]:
                    f.append(("gyrotaxis_velocity", "gyrotaxis_velocity"))
            if flags2 & abi.FLAGS2["LAGRANGE_ORIENTATION_ACTIVE"]:
                f.append(("swim_velocity", "swim_velocity"))
                if flags2 & abi.FLAGS2["LAGRANGE_ORIENTATION_ACTIVE_JUMP"]:  # src/lagrange.c:1993-2011
                    f += [(n, n) for n in ("critical_shear_rate", "shear_rate", "jump_time")]
    if flags & abi.FLAGS["LB_TEMPERATURE"]:
        f += [("temperature", "t"), ("dt_t", "dt_t")]
        if grad:
            f += [("dx_t", "dx_t"), ("dy_t", "dy_t"), ("dz_t", "dz_t")]
        if flags2 & abi.FLAGS2["LAGRANGE_TEMPERATURE"]:
            f += [("temperature_particle", "t_p"), ("cp_particle", "cp_p")]
    return f


def _particle_sim(name, seed, nsteps):
    _, cfg, state = make_case(name, seed=seed)
    sim = ch4b200.Simulation(cfg)
    for k, v in pop_items(state):
        sim.set_pop(k, v)
    sim.set_particles(state["part"])
    sim.initialize()
    sim.step(nsteps)
    return cfg, state, sim


@pytest.mark.parametrize("name", ["particles", "particles_t", "particles_or", "particles_tt", "particles_swims",
                                  "particles_swimt", "particles_jump"])
def test_particle_file_holds_the_particles(name, tmp_path):
    cfg, state, sim = _particle_sim(name, 65, 4)
    with sim:
        n = len(state["part"])
        sim.output_particles_h5(tmp_path, 4, time_now=4.0, output_fluid=True)
        parts = sim.get_particles(n)
    got = h5spec.read(tmp_path / "particle_4.h5")
    want = _fields(cfg.flags, True, cfg.flags2)
    assert sorted(k for k in got) == sorted("/lagrange/" + d for d, _ in want)
    for d, field in want:
        assert np.array_equal(got["/lagrange/" + d], np.array([getattr(p, field) for p in parts])), d
    xmf = (tmp_path / "particle_4.xmf").read_text()
    assert '<Topology TopologyType="Polyvertex" NumberOfElements="%d"/>' % n in xmf
    for d, _ in want:
        assert "particle_4.h5:/lagrange/%s\n" % d in xmf, d


@pytest.mark.parametrize("name", ["particles", "particles_t", "particles_or", "particles_tt", "particles_swims"])
def test_part_file_restart(name, tmp_path):
    cfg, state, a = _particle_sim(name, 66, 5)
    n = len(state["part"])
    with a:
        a.write_pop_h5(tmp_path / "pop.h5")
        a.write_particles_h5(tmp_path / "part.h5")
        pops = {k: a.get_pop(k) for k, _ in pop_items(state)}
        parts = a.get_particles(n)
        phases = a.get_hit_phases()
    got = h5spec.read(tmp_path / "part.h5")
    rec = got["/particles/point_particle"]
    members = rec.dtype.names
    assert members[:17] == ("name", "x", "y", "z", "vx", "vy", "vz", "vx_old", "vy_old", "vz_old", "ax", "ay",
                            "az", "ax_old", "ay_old", "az_old", "tau_drag")
    assert ("t" in members) == bool(cfg.flags & abi.FLAGS["LB_TEMPERATURE"])
    field = {"temperature_particle": "t_p", "cp_particle": "cp_p"}  # member name -> ch4_particle field
    for m in members:
        assert np.array_equal(rec[m], np.array([getattr(p, field.get(m, m)) for p in parts])), m
    assert got["/properties@particle_types"].item() == float(cfg.particle_types)
    # the members part.h5 lacks start at 0, as in the reference's resume
    trimmed = (ch4b200.Particle * n)()
    for i, p in enumerate(parts):
        for m in members:
            setattr(trimmed[i], field.get(m, m), getattr(p, field.get(m, m)))
    with ch4b200.Simulation(cfg) as b, ch4b200.Simulation(cfg) as c:
        b.read_pop_h5(tmp_path / "pop.h5")
        b.read_particles_h5(tmp_path / "part.h5")
        for k, arr in pops.items():
            c.set_pop(k, arr)
        c.set_particles(trimmed)
        if cfg.flags & abi.FLAGS["LB_FLUID_FORCING_HIT"]:  # pop.h5 carries the phases
            c.set_hit_phases(phases)
        back = b.get_particles(n)
        for m in (f for f, _ in ch4b200.Particle._fields_):
            assert np.array_equal([getattr(p, m) for p in back], [getattr(p, m) for p in trimmed]), m
        b.initialize()
        c.initialize()
        b.step(3)
        c.step(3)
        pb, pc = b.get_particles(n), c.get_particles(n)
        for m in ("x", "y", "z", "vx", "vy", "vz", "px", "py", "pz"):
            assert np.array_equal([getattr(p, m) for p in pb], [getattr(p, m) for p in pc]), m
        if cfg.flags & abi.FLAGS["LAGRANGE_ORIENTATION"]:  # the orientation survives the restart
            assert np.isfinite([p.px for p in pb]).all()
            assert np.array_equal(rec["aspect_ratio"], [p.aspect_ratio for p in parts])
