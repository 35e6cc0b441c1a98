"""Host-side checks that need no GPU: the C ABI library loads and exports every
symbol include/ch4.h declares; the define.h / param.in readers follow the
reference's semantics (src/parameters.c:3-39)."""
import os
import re

import pytest

import ch4b200
from ch4b200 import abi

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(REPO, "include", "ch4.h")).read()
    return sorted(set(re.findall(r"^(?:ch4_status|const char \*)\s*(ch4_\w+)\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    L = ch4b200.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n


def test_config_default():
    c = ch4b200.default_config()
    assert c.C_smag == 0.18 and c.time_dt == 1.0 and c.flags == abi.FLAGS["LB_FLUID"]


def test_read_param_semantics(tmp_path):
    p = tmp_path / "param.in"
    # first number after a key wins; extra numbers are consumed as junk pairs
    p.write_text("resume 0\nNX 16\nNY 8\nNZ 4\nSX 16\nSY 8\nSZ 4\ntime_dt 1.0\n"
                 "tau_u 0.6 0.51 0.52 0.53 0.54\nAmp_x 1.e-2\nAmp_y 0\nAmp_z 0\n")
    c = ch4b200.default_config()
    c.flags = abi.flags_of(["LB_FLUID", "LB_FLUID_FORCING"])
    ch4b200.read_param(c, str(p))
    assert (c.NX, c.NY, c.NZ) == (16, 8, 4)
    assert c.tau_u == 0.6 and c.Amp_x == 1e-2
    assert c.nu == (0.6 - 0.5 * 1.0) / 3.0
    assert ch4b200.read_parameter(str(p), "tau_u") == 0.6


def test_read_param_missing_key(tmp_path):
    p = tmp_path / "param.in"
    p.write_text("resume 0\nNX 16\nNY 8\n")
    c = ch4b200.default_config()
    with pytest.raises(ch4b200.CH4Error) as e:
        ch4b200.read_param(c, str(p))
    assert e.value.status == abi.ERR_PARAM and "NZ" in str(e.value)


def test_read_define(tmp_path):
    d = tmp_path / "define.h"
    d.write_text("#define SYSTEM_RANDOM48\n//#define LB_SCALAR\n#define GRID_POP_D3Q19\n#define LB\n#define LB_FLUID\n"
                 "#define LB_FLUID_FORCING /* force */\n#define LB_FLUID_FORCING_KOLMOGOROV\n#define METHOD_STREAMING\n"
                 "/* #define LB_TEMPERATURE */\n#define LB_TEMPERATURE_BUOYANCY_T0_REF\n")
    c = ch4b200.default_config()
    ch4b200.read_define(c, str(d))
    assert abi.set_flag_names(c.flags) == ["LB_FLUID", "LB_FLUID_FORCING", "LB_FLUID_FORCING_KOLMOGOROV"]
    assert c.t0_kind == abi.T0_REF


def test_read_define_rejects_out_of_scope_flag(tmp_path):
    d = tmp_path / "define.h"
    d.write_text("#define GRID_POP_D3Q19\n#define METHOD_STREAMING\n#define LB_TEMPERATURE_MELTING\n")
    c = ch4b200.default_config()
    with pytest.raises(ch4b200.CH4Error) as e:
        ch4b200.read_define(c, str(d))
    assert e.value.status == abi.ERR_UNSUPPORTED and "LB_TEMPERATURE_MELTING" in str(e.value)


def test_read_define_requires_d3q19_streaming(tmp_path):
    d = tmp_path / "define.h"
    d.write_text("#define GRID_POP_D2Q9\n#define METHOD_STREAMING\n")
    with pytest.raises(ch4b200.CH4Error):
        ch4b200.read_define(ch4b200.default_config(), str(d))


def test_device_bytes_admission():
    c = ch4b200.default_config()
    c.NX, c.NY, c.NZ = 256, 256, 128
    c.SX, c.SY, c.SZ = 256.0, 256.0, 128.0
    c.flags = abi.flags_of(["LB_FLUID", "LB_TEMPERATURE"])
    c.storage = abi.STORE_F32
    n = ch4b200.device_bytes(c)
    cells = 256 * 256 * 128
    assert n >= 2 * 2 * 19 * cells * 4
    c.storage = abi.STORE_F16
    assert ch4b200.device_bytes(c) < n


def test_walls_on_x_and_z_are_read_from_define_h(tmp_path):
    """LB_FLUID_BC_X / _Z, the temperature and scalar walls on x and z and the wall
    umbrellas land in the second flag word."""
    import ch4b200
    from ch4b200 import abi
    d = tmp_path / "define.h"
    d.write_text("#define GRID_POP_D3Q19\n#define METHOD_STREAMING\n#define LB_FLUID\n#define LB_FLUID_BC\n"
                 "#define LB_FLUID_BC_X\n#define LB_FLUID_BC_Z\n#define LB_FLUID_BC_Z_P_SLIP\n"
                 "#define LB_TEMPERATURE\n#define LB_TEMPERATURE_BC_X\n#define LB_TEMPERATURE_BC_X_M_NOFLUX\n")
    c = ch4b200.default_config()
    ch4b200.read_define(c, str(d))
    assert c.flags2 == abi.flags2_of(["LB_FLUID_BC", "LB_FLUID_BC_X", "LB_FLUID_BC_Z", "LB_FLUID_BC_Z_P_SLIP",
                                      "LB_TEMPERATURE_BC_X", "LB_TEMPERATURE_BC_X_M_NOFLUX"])
    assert abi.has_flag(c, "LB_FLUID_BC_X") and not abi.has_flag(c, "LB_FLUID_BC_Y")


@pytest.mark.parametrize("names", [
    ["LB_FLUID", "LB_FLUID_BC_X", "LB_FLUID_BC_Z", "LB_FLUID_BC_Z_P_SLIP"],
    ["LB_FLUID", "LB_FLUID_BC_Y", "LB_FLUID_BC_Y_M_SLIP", "LB_FLUID_BC_X"],
    ["LB_FLUID", "LB_FLUID_BC_X_P_SLIP"],
])
def test_slip_wall_beside_another_wall_is_refused(names):
    """Checked before any device call: a slip wall needs every other axis periodic, and
    a slip flag needs its axis's walls."""
    import ctypes as C
    c = ch4b200.default_config()
    c.NX, c.NY, c.NZ = 6, 5, 4
    c.SX, c.SY, c.SZ = 6.0, 5.0, 4.0
    c.tau_u = 0.6
    abi.set_flags(c, names)
    h = C.c_void_p()
    rc = ch4b200.lib().ch4_create(C.byref(c), C.byref(h))
    assert rc in (abi.ERR_UNSUPPORTED, abi.ERR_ARG) and not h.value


def test_particle_wall_and_small_tau_flags_are_read_from_define_h(tmp_path):
    """The particles' wall rules and small-tau_drag models are flags of the second word;
    the beta small-tau_drag model without added mass and gradients is refused at create."""
    import ctypes as C
    d = tmp_path / "define.h"
    d.write_text("#define GRID_POP_D3Q19\n#define METHOD_STREAMING\n#define LB_FLUID\n#define LB_FLUID_BC\n"
                 "#define LB_FLUID_BC_Y\n#define LAGRANGE\n#define LAGRANGE_WRAP\n#define LAGRANGE_BC_INELASTIC\n"
                 "#define LAGRANGE_BC_INELASTIC_REINJECT\n#define LAGRANGE_SMALLTAUD\n"
                 "#define LAGRANGE_SMALLTAUD_BETA\n#define LAGRANGE_TWOWAY_SMALLTAUD\n")
    c = ch4b200.default_config()
    ch4b200.read_define(c, str(d))
    assert abi.has_flag(c, "LAGRANGE_BC_INELASTIC_REINJECT") and abi.has_flag(c, "LAGRANGE_SMALLTAUD_BETA")
    assert abi.has_flag(c, "LB_FLUID_BC") and abi.has_flag(c, "LAGRANGE_TWOWAY_SMALLTAUD")
    c.NX, c.NY, c.NZ = 6, 5, 4
    c.SX, c.SY, c.SZ = 6.0, 5.0, 4.0
    c.tau_u, c.time_dt, c.time_dt_lagr_factor = 0.6, 1.0, 1.0
    h = C.c_void_p()
    assert ch4b200.lib().ch4_create(C.byref(c), C.byref(h)) == abi.ERR_UNSUPPORTED and not h.value


@pytest.mark.parametrize("flagset", ["particles_orbc", "particles_sed", "particles_rad"])
def test_particle_wall_variants_read_from_the_oracle_define_h(flagset):
    """The define.h of each particle-wall variant gives the flag words the oracle runs."""
    import oracle as O
    c = ch4b200.default_config()
    ch4b200.read_define(c, os.path.join(REPO, "oracle", "configs", flagset + ".h"))
    names = O.FLAGSETS[flagset]
    assert all(abi.has_flag(c, n) for n in names)
    assert int(c.flags2) & ~sum(abi.FLAGS2[n] for n in names if n in abi.FLAGS2) == 0


def test_param_reader_radius_density_types_and_time_start(tmp_path):
    """LAGRANGE_RADIUSandDENSITY counts the types by radius and density instead of tau_drag and
    beta (src/parameters.c:530-556); GRAVITY_VARIABLE multiplies them by the gravity classes
    (src/parameters.c:590-602); time_start starts the step clock (src/parameters.c:138-140)."""
    p = tmp_path / "param.in"
    p.write_text("resume 0\nNX 8\nNY 8\nNZ 8\nSX 8\nSY 8\nSZ 8\ntime_dt 1.0\ntime_start 2.5\ntau_u 0.6\n"
                 "gravity_x 0\ngravity_y 1e-3\ngravity_z 0\ntime_dt_lagr_factor 1\nparticle_number 10\n"
                 "tau_drag_types 7\nbeta_coeff_types 5\nparticle_radius_types 2\nparticle_density_types 3\n"
                 "gravity_coeff_types 4\n")
    c = ch4b200.default_config()
    c.flags = abi.flags_of(["LB_FLUID", "LAGRANGE", "LAGRANGE_GRADIENT", "LAGRANGE_ADDEDMASS", "LAGRANGE_GRAVITY"])
    ch4b200.read_param(c, str(p))
    assert c.particle_types == 7 * 5 and c.time_start == 2.5
    c.flags2 = abi.FLAGS2["LAGRANGE_RADIUSandDENSITY"] | abi.FLAGS2["LAGRANGE_GRAVITY_VARIABLE"]
    ch4b200.read_param(c, str(p))
    assert c.particle_types == 2 * 3 * 4
