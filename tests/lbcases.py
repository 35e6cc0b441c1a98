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
}


def make_case(name, seed=0, storage=0, **over):
    c = dict(CASES[name])
    params = dict(c["params"])
    params.update(over)
    flags = O.FLAGSETS[c["flagset"]]
    params.update(O.FLAGSET_EXTRA.get(c["flagset"], {}))
    cfg = O.make_config(c["NX"], c["NY"], c["NZ"], flags, storage=storage, **params)
    rng = np.random.default_rng(seed)
    state = {"p": pops(rng, c["NX"], c["NY"], c["NZ"], 1.0, 3e-2 if name == "les" else 1e-2)}
    if "LB_TEMPERATURE" in flags:
        state["g"] = rb_temperature_pops(rng, c["NX"], c["NY"], c["NZ"], cfg.T_bot, cfg.T_top, 1e-2)
    if "LB_SCALAR" in flags:
        state["h"] = pops(rng, c["NX"], c["NY"], c["NZ"], 0.3, 1e-1)
    return c["flagset"], cfg, state


def run_restatement(cfg, state, nsteps, phi=None):
    r = O.Restatement(cfg)
    for k, v in state.items():
        r.set_pop(k, v)
    if phi is not None:
        r.set_hit_phases(phi)
    r.initialize()
    r.step(nsteps)
    out = {k: r.get_pop(k) for k in state}
    out.update(r.fields())
    out["force"] = r.force()
    if cfg.flags & O.abi.FLAGS["LB_FLUID_FORCING_HIT"]:
        out["phi"] = r.get_hit_phases()
    r.close()
    return out
