"""Seeded lattice cases shared by the oracle pin tests and the GPU parity tests.

Each case names a compiled reference flag set (oracle/configs/<flagset>.h), the
matching product flags, the param.in values and the initial populations (seeded
perturbations of the rest state, injected through the reference's restart-free
path).  Sizes are small enough for the CPU oracle to finish in well under a second.
"""
import numpy as np

import oracle as O

W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def pops(rng, NX, NY, NZ, base, amp):
    return (base * W)[None, None, None, :] * (1 + amp * rng.standard_normal((NZ, NY, NX, 19)))


def rb_temperature_pops(rng, NX, NY, NZ, T_bot, T_top, amp):
    """Linear conductive profile (src/initial_conditions.c:303-308) + seeded noise."""
    y = (np.arange(NY) + 0.5) / NY
    T = T_bot + (T_top - T_bot) * y
    T = T[None, :, None] + amp * (2 * rng.random((NZ, NY, NX)) - 1)
    return T[..., None] * W[None, None, None, :]


CASES = {
    "kolmogorov": dict(flagset="kolmogorov", NX=8, NY=6, NZ=5,
                       params=dict(tau_u=0.6, Amp_x=0.01, Amp_y=0.002, Amp_z=0.003)),
    "rb": dict(flagset="rb", NX=8, NY=7, NZ=5,
               params=dict(tau_u=0.55, tau_t=0.57, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.3,
                           gravity_y=1e-3, gravity_x=2e-4)),
    "hit": dict(flagset="hit", NX=8, NY=7, NZ=6,
                params=dict(tau_u=0.56, Amp_x=2e-4, Amp_y=1.5e-4, Amp_z=1e-4, seed=4)),
    "walls2": dict(flagset="walls2", NX=7, NY=6, NZ=5,
                   params=dict(tau_u=0.62, tau_t=0.58, T_bot=1.0, T_top=-0.5, T_ref=0.2, beta_t=0.2,
                               beta2_t=0.05, gravity_y=2e-3, gravity_z=-3e-4, Amp_x=2e-3, grad_T_top=-0.03,
                               grad_T_bot=0.01)),
    "scalar": dict(flagset="scalar", NX=6, NY=8, NZ=5,
                   params=dict(tau_u=0.6, tau_t=0.65, tau_s=0.7, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.2,
                               S_bot=0.2, S_top=0.7, S_ref=0.1, beta_s=0.3, gravity_y=2e-3, gravity_x=1e-3)),
    "les": dict(flagset="les", NX=8, NY=9, NZ=6,
                params=dict(tau_u=0.52, Amp_x=0.02, Amp_y=0.01, Amp_z=0.005)),
    "les_sism": dict(flagset="les_sism", NX=8, NY=9, NZ=6,
                     params=dict(tau_u=0.52, Amp_x=0.02, Amp_y=0.01, Amp_z=0.005)),
    "les_kalman": dict(flagset="les_kalman", NX=8, NY=9, NZ=6,
                       params=dict(tau_u=0.52, Amp_x=0.02, Amp_y=0.01, Amp_z=0.005)),
    "les_vd": dict(flagset="les_vd", NX=8, NY=12, NZ=6,
                   params=dict(tau_u=0.52, Amp_x=0.02, Amp_y=0.01, Amp_z=0.005)),
    "les_ls": dict(flagset="les_ls", NX=8, NY=9, NZ=6,
                   params=dict(tau_u=0.52, Amp_x=0.02, Amp_y=0.01, Amp_z=0.005)),
    "les_wale": dict(flagset="les_wale", NX=8, NY=9, NZ=6,
                     params=dict(tau_u=0.52, Amp_x=0.02, Amp_y=0.01, Amp_z=0.005)),
    "les_ts": dict(flagset="les_ts", NX=6, NY=8, NZ=5,
                   params=dict(tau_u=0.53, tau_t=0.56, tau_s=0.58, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.2,
                               S_bot=0.2, S_top=0.7, S_ref=0.1, beta_s=0.3, gravity_y=2e-3, gravity_x=1e-3)),
    "trt": dict(flagset="trt", NX=8, NY=7, NZ=5,
                params=dict(tau_u=0.62, tau_t=0.7, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.3,
                            gravity_y=1e-3, gravity_x=2e-4)),
    "trt_les": dict(flagset="trt_les", NX=8, NY=9, NZ=6,
                    params=dict(tau_u=0.52, Amp_x=0.02, Amp_y=0.01, Amp_z=0.005)),
    "particles": dict(flagset="particles", NX=10, NY=8, NZ=7, npart=300,
                      params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=6,
                                  time_dt_lagr_factor=2.0, particle_number=300)),
    "nozero": dict(flagset="nozero", NX=8, NY=7, NZ=6,
                   params=dict(tau_u=0.58, tau_t=0.62, Amp_x=3e-3, Amp_y=1e-3, Amp_z=2e-3, T_bot=1.0, T_top=0.0,
                               T_ref=0.5, beta_t=0.3, gravity_y=2e-3, gravity_x=1e-3)),
    "cpower": dict(flagset="cpower", NX=8, NY=7, NZ=6,
                   params=dict(tau_u=0.57, Amp_x=1e-9, Amp_y=8e-10, Amp_z=5e-10, seed=3)),
    "particles_tc": dict(flagset="particles_tc", NX=10, NY=8, NZ=7, npart=300,
                         params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=9,
                                     time_dt_lagr_factor=2.0, particle_number=300)),
    "particles_or": dict(flagset="particles_or", NX=10, NY=8, NZ=7, npart=300,
                         params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=4,
                                     time_dt_lagr_factor=2.0, particle_number=300)),
    "particles_1w": dict(flagset="particles_1w", NX=10, NY=8, NZ=7, npart=300,
                         params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=8,
                                     time_dt_lagr_factor=2.0, particle_number=300)),
    "particles_g": dict(flagset="particles_g", NX=10, NY=8, NZ=7, npart=300,
                        params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=7, gravity_x=2e-5,
                                    gravity_y=1e-4, gravity_z=-3e-5, time_dt_lagr_factor=2.0, particle_number=300)),
    "particles_t": dict(flagset="particles_t", NX=9, NY=8, NZ=7, npart=250,
                        params=dict(tau_u=0.56, tau_t=0.6, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=5,
                                    T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.2, gravity_y=1e-3,
                                    time_dt_lagr_factor=2.0, particle_number=250)),
    # particles with their own temperature, coupled back through momentum and heat
    "particles_tt": dict(flagset="particles_tt", NX=9, NY=8, NZ=7, npart=250,
                         params=dict(tau_u=0.56, tau_t=0.6, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=12,
                                     T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.2, gravity_y=1e-3,
                                     time_dt_lagr_factor=2.0, particle_number=250)),
    "particles_ttc": dict(flagset="particles_ttc", NX=9, NY=8, NZ=7, npart=250,
                          params=dict(tau_u=0.56, tau_t=0.6, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=13,
                                      T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.2, gravity_y=1e-3,
                                      time_dt_lagr_factor=2.0, particle_number=250)),
    # particles in wall-bounded flows
    "particles_rb": dict(flagset="particles_rb", NX=9, NY=8, NZ=7, npart=250,
                         params=dict(tau_u=0.56, tau_t=0.6, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.3,
                                     gravity_y=1e-3, gravity_x=2e-4, seed=14, time_dt_lagr_factor=2.0,
                                     particle_number=250)),
    "particles_duct": dict(flagset="particles_duct", NX=10, NY=8, NZ=7, npart=300,
                           params=dict(tau_u=0.6, Amp_x=4e-3, Amp_y=1e-3, Amp_z=2e-3, seed=15,
                                       time_dt_lagr_factor=2.0, particle_number=300)),
    "particles_slip": dict(flagset="particles_slip", NX=8, NY=7, NZ=6, npart=250,
                           params=dict(tau_u=0.57, tau_t=0.61, T_bot=0.3, T_top=1.0, T_ref=0.5, Amp_x=2e-3,
                                       Amp_y=1e-3, Amp_z=5e-4, seed=16, time_dt_lagr_factor=2.0,
                                       particle_number=250)),
    "particles_reinj": dict(flagset="particles_reinj", NX=9, NY=8, NZ=7, npart=250,
                            params=dict(tau_u=0.56, tau_t=0.6, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.3,
                                        gravity_y=1e-3, gravity_x=2e-4, gravity_z=-1e-4, seed=17,
                                        time_dt_lagr_factor=2.0, particle_number=250)),
    "particles_rjr": dict(flagset="particles_rjr", NX=9, NY=8, NZ=7, npart=250,
                          params=dict(tau_u=0.56, tau_t=0.6, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.3,
                                      gravity_y=1e-3, gravity_x=2e-4, gravity_z=-1e-4, seed=19,
                                      time_dt_lagr_factor=2.0, particle_number=250)),
    "particles_sed": dict(flagset="particles_sed", NX=9, NY=8, NZ=7, npart=250,
                          params=dict(tau_u=0.56, tau_t=0.6, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.3,
                                      gravity_y=1e-3, gravity_x=2e-4, seed=21, time_dt_lagr_factor=2.0,
                                      particle_number=250, time_start=2.5)),
    "particles_rad": dict(flagset="particles_rad", NX=9, NY=8, NZ=7, npart=250,
                          params=dict(tau_u=0.56, tau_t=0.6, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.3,
                                      gravity_y=1e-3, gravity_x=2e-4, seed=22, time_dt_lagr_factor=2.0,
                                      particle_number=250)),
    "particles_orbc": dict(flagset="particles_orbc", NX=9, NY=8, NZ=7, npart=250,
                           params=dict(tau_u=0.56, tau_t=0.6, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.3,
                                       gravity_y=1e-3, gravity_x=2e-4, seed=20, time_dt_lagr_factor=2.0,
                                       particle_number=250)),
    "particles_bc": dict(flagset="particles_bc", NX=9, NY=8, NZ=7, npart=250,
                         params=dict(tau_u=0.56, tau_t=0.6, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=18,
                                     T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.2, gravity_y=1e-3, gravity_x=3e-4,
                                     time_dt_lagr_factor=2.0, particle_number=250)),
    # orientation variants and swimming tracers
    "particles_or2": dict(flagset="particles_or2", NX=10, NY=8, NZ=7, npart=300,
                          params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=21, gravity_x=2e-5,
                                      gravity_y=1e-4, gravity_z=-3e-5, time_dt_lagr_factor=2.0, particle_number=300)),
    "particles_swimt": dict(flagset="particles_swimt", NX=9, NY=8, NZ=7, npart=250,
                            params=dict(tau_u=0.56, tau_t=0.6, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=22,
                                        T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.2, gravity_y=1e-3,
                                        time_dt_lagr_factor=2.0, particle_number=250)),
    "particles_swimb": dict(flagset="particles_swimb", NX=10, NY=8, NZ=7, npart=300,
                            params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=23,
                                        time_dt_lagr_factor=2.0, particle_number=300)),
    "particles_swims": dict(flagset="particles_swims", NX=10, NY=8, NZ=7, npart=300,
                            params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=24,
                                        time_dt_lagr_factor=2.0, particle_number=300)),
    "particles_swimn": dict(flagset="particles_swimn", NX=10, NY=8, NZ=7, npart=300,
                            params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=25,
                                        time_dt_lagr_factor=2.0, particle_number=300)),
    # orientation noise drawn from the drand48 stream, with HIT phase walks in between
    "particles_rdiff": dict(flagset="particles_rdiff", NX=10, NY=8, NZ=7, npart=300,
                            params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=26,
                                        time_dt_lagr_factor=2.0, particle_number=300)),
    "particles_rand": dict(flagset="particles_rand", NX=9, NY=10, NZ=6, npart=200,
                           params=dict(tau_u=0.6, Amp_x=3e-3, seed=27, time_dt_lagr_factor=3.0, particle_number=200)),
    # run-and-tumble swimmers
    "particles_jump": dict(flagset="particles_jump", NX=10, NY=8, NZ=7, npart=300,
                           params=dict(tau_u=0.55, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=28,
                                       time_dt_lagr_factor=2.0, particle_number=300)),
    "particles_jumpt": dict(flagset="particles_jumpt", NX=9, NY=8, NZ=7, npart=250,
                            params=dict(tau_u=0.56, tau_t=0.6, Amp_x=2e-3, Amp_y=1.5e-3, Amp_z=1e-3, seed=29,
                                        T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.2, gravity_y=1e-3,
                                        time_dt_lagr_factor=2.0, particle_number=250)),
    # Smagorinsky-Lilly: T rising with y (stable), so the buoyancy damps |S| where Ri < 1
    "les_lilly": dict(flagset="les_lilly", NX=8, NY=9, NZ=6,
                      params=dict(tau_u=0.52, tau_t=0.55, Amp_x=0.02, T_bot=0.0, T_top=1.0, T_ref=0.5, beta_t=0.3,
                                  gravity_y=1e-3, gravity_x=0.0)),
    # walls on x and z
    "duct": dict(flagset="duct", NX=7, NY=8, NZ=6,
                 params=dict(tau_u=0.6, Amp_x=4e-3, Amp_y=1e-3, Amp_z=2e-3)),
    "duct_les": dict(flagset="duct_les", NX=8, NY=9, NZ=7,
                     params=dict(tau_u=0.52, Amp_x=0.02, Amp_y=0.01, Amp_z=0.005)),
    "box": dict(flagset="box", NX=7, NY=8, NZ=6,
                params=dict(tau_u=0.58, tau_t=0.62, tau_s=0.66, T_bot=1.0, T_top=0.0, T_ref=0.5, beta_t=0.3,
                            S_bot=0.2, S_top=0.7, S_ref=0.1, beta_s=0.2, gravity_y=2e-3, gravity_x=5e-4,
                            gravity_z=-3e-4)),
    "slipx": dict(flagset="slipx", NX=8, NY=6, NZ=5,
                  params=dict(tau_u=0.57, tau_t=0.61, T_bot=0.3, T_top=1.0, T_ref=0.5, beta_t=0.3,
                              gravity_x=2e-3, gravity_y=7e-4)),
    "slipz": dict(flagset="slipz", NX=6, NY=5, NZ=8,
                  params=dict(tau_u=0.59, tau_t=0.63, tau_s=0.6, T_bot=1.0, T_top=0.1, T_ref=0.5, beta_t=0.25,
                              S_bot=0.4, S_top=0.9, S_ref=0.2, gravity_z=2e-3, gravity_x=6e-4)),
}


def make_particles(rng, n, NX, NY, NZ):
    """Tracers and Stokes particles (beta in {1, 3}, tau_drag in {0.5, 2, 5}), uniform
    random positions (a few exactly on cell centres and faces), at rest."""
    from ch4b200 import abi
    parts = (abi.Particle * n)()
    taus = [0.0, 0.5, 2.0, 5.0]
    betas = [1.0, 3.0]
    for i in range(n):
        p = parts[i]
        p.name = float(i)
        p.tau_drag = taus[i % len(taus)]
        p.beta_coeff = betas[(i // len(taus)) % len(betas)]
        p.x, p.y, p.z = rng.random() * NX, rng.random() * NY, rng.random() * NZ
        if i % 50 == 7:  # on a cell centre / on the domain face
            p.x, p.y, p.z = 0.5 + (i % NX), 0.0, float(NZ) - 0.5
    return parts


def make_case(name, seed=0, storage=0, dims=None, **over):
    """(flagset, config, initial state) of a case; `dims` = (NX, NY, NZ) overrides its lattice."""
    c = dict(CASES[name])
    if dims is not None:
        c["NX"], c["NY"], c["NZ"] = dims
    params = dict(c["params"])
    params.update(over)
    flags = O.FLAGSETS[c["flagset"]]
    params.update(O.FLAGSET_EXTRA.get(c["flagset"], {}))
    cfg = O.make_config(c["NX"], c["NY"], c["NZ"], flags, storage=storage, **params)
    rng = np.random.default_rng(seed)
    state = {"p": pops(rng, c["NX"], c["NY"], c["NZ"], 1.0, 3e-2 if name in ("les", "les_lilly") else 1e-2)}
    if "LB_TEMPERATURE" in flags:
        state["g"] = rb_temperature_pops(rng, c["NX"], c["NY"], c["NZ"], cfg.T_bot, cfg.T_top, 1e-2)
    if "LB_SCALAR" in flags:
        state["h"] = pops(rng, c["NX"], c["NY"], c["NZ"], 0.3, 1e-1)
    if "LAGRANGE" in flags:
        state["part"] = make_particles(rng, c["npart"], c["NX"], c["NY"], c["NZ"])
        if "LAGRANGE_TEMPERATURE" in flags:
            # inertial particles only (the thermal relaxation and exchange rates divide by
            # tau_drag and beta), specific heats 0.5 .. 2, temperatures about the fluid's
            cps = [0.5, 1.0, 2.0]
            for i, p in enumerate(state["part"]):
                p.tau_drag = [0.5, 2.0, 5.0][i % 3]
                p.beta_coeff = [1.0, 2.0, 0.5][(i // 3) % 3]  # 3 - beta divides the heat rate
                p.cp_p = cps[(i // 9) % 3]
                p.t_p = 0.3 + 0.4 * rng.random()
        walls = [a for a, w in enumerate(("LB_FLUID_BC_X", "LB_FLUID_BC_Y", "LB_FLUID_BC_Z")) if w in flags]
        if walls:
            # every fifth particle starts a hair inside a wall, moving out through it
            # (inertial particles keep that velocity into their first sub-step)
            size = (c["NX"], c["NY"], c["NZ"])
            for i, p in enumerate(state["part"]):
                if i % 5 != 2:
                    continue
                a = walls[(i // 5) % len(walls)]
                upper = (i // 10) % 2 == 1
                pos = size[a] - 1e-3 * (1 + i % 7) if upper else 1e-3 * (1 + i % 7)
                vel = 0.02 * (1 + i % 3) * (1 if upper else -1)
                setattr(p, "xyz"[a], pos)
                setattr(p, "v" + "xyz"[a], vel)
        if "LAGRANGE_ORIENTATION" in flags:  # random unit orientations, rods and discs
            ratios = [1.0, 5.0, 0.2, 20.0]
            for i, p in enumerate(state["part"]):
                v = rng.normal(size=3)
                p.px, p.py, p.pz = v / np.linalg.norm(v)
                p.aspect_ratio = ratios[i % len(ratios)]
        if "LAGRANGE_ORIENTATION_SECONDORIENTATION" in flags:  # a second random unit vector
            for p in state["part"]:
                v = rng.normal(size=3)
                p.nx, p.ny, p.nz = v / np.linalg.norm(v)
        if "LAGRANGE_ORIENTATION_JEFFREY_GYROTAXIS" in flags:  # 0 switches the term off
            for i, p in enumerate(state["part"]):
                p.gyrotaxis_velocity = [0.0, 0.5, 2.0, -1.0, 10.0][i % 5]
        if "LAGRANGE_ORIENTATION_ACTIVE" in flags:
            for i, p in enumerate(state["part"]):
                p.swim_velocity = [0.01, 0.0, 0.03, 0.002][(i // 4) % 4]
        if "LAGRANGE_ORIENTATION_ACTIVE_JUMP" in flags:  # thresholds either side of the flow's values
            crit = ([0.3, 0.5, 0.7, 1e10] if "LAGRANGE_ORIENTATION_ACTIVE_JUMP_TEMPERATURE" in flags
                    else [1e-5, 1e-4, 1e-3, 1e10])
            for i, p in enumerate(state["part"]):
                p.critical_shear_rate = crit[i % 4]
                p.jump_time = [0.0, 0.5, 2.0, 5.0][(i // 4) % 4]
                p.time_from_jump = [0.0, 0.3, 3.0, 30.0][(i // 16) % 4]
                v = rng.normal(size=3)
                p.px_jump, p.py_jump, p.pz_jump = v / np.linalg.norm(v)
        if "LAGRANGE_ORIENTATION_DIFFUSION" in flags:  # 0 for some: their p is still normalised
            for i, p in enumerate(state["part"]):
                p.rotational_diffusion = [0.0, 0.01, 0.1, 0.002][(i // 2) % 4]
        if "LAGRANGE_GRAVITY_VARIABLE" in flags:  # gravity off, scaled down and up; earlier depositions
            for i, p in enumerate(state["part"]):
                p.gravity_coeff = [1.0, 0.0, 0.3, 2.5][i % 4]
                p.sediment = [0.0, 0.0, 3.0, 1.25][(i // 4) % 4]
    return c["flagset"], cfg, state


def pop_items(state):
    return [(k, v) for k, v in state.items() if k in ("p", "g", "h")]


def run_restatement(cfg, state, nsteps, phi=None):
    r = O.Restatement(cfg)
    for k, v in pop_items(state):
        r.set_pop(k, v)
    if "part" in state:
        r.set_particles(state["part"])
    if phi is not None:
        r.set_hit_phases(phi)
    r.initialize()
    r.step(nsteps)
    out = {k: r.get_pop(k) for k, _ in pop_items(state)}
    if "part" in state:
        out["part"] = O.particles_as_dict(r.get_particles(len(state["part"])))
    out.update(r.fields())
    out["force"] = r.force()
    out["avg"] = r.averages()
    if cfg.flags & O.abi.FLAGS["LB_FLUID_FORCING_HIT"]:
        out["phi"] = r.get_hit_phases()
    r.close()
    return out
