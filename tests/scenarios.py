"""Small seeded scenes for parity tests (sizes the reference finishes in
seconds).  Each entry: (scene spec factory, steps, dump steps)."""
import math

from peridem_b200 import scene

R = 1e-3


def two_particle_rnp():
    # top disc 0.02 h above first contact, approaching at 1 m/s
    return scene.two_particle(h_div=10, radius=R, material="RNPBond", v0=-1.0, gap=0.02 * R / 10,
                              nt=400)


def two_particle_pmb_impact():
    # fast impact that breaks bonds (PMB, bond breaking by critical stretch)
    return scene.two_particle(h_div=8, radius=R, material="PMBBond", v0=-40.0, gap=0.01 * R / 8,
                              nt=300)


def two_particle_state():
    return scene.two_particle(h_div=8, radius=R, material="PDState", v0=-2.0, gap=0.02 * R / 8,
                              nt=300)


def two_particle_verlet():
    s = scene.two_particle(h_div=8, radius=R, material="RNPBond", v0=-1.0, gap=0.02 * R / 8, nt=200)
    s.time_scheme = "velocity_verlet"
    return s


def compressive_small():
    h = R / 6
    return scene.compressive_2d(n_particles=6, r_range=(R, 1.2 * R), h_div=6, width=8e-3, seed=3,
                                gap=1.02 * h, wall_speed=-2.0, nt=400, search_interval=10)


def column_3d_small():
    return scene.column_3d(n_spheres=2, median_r=R, sigma=0.0, h_div=4, box=(3e-3, 3e-3, 6e-3),
                           seed=1, material="PDState", piston_speed=-2.0, nt=200)


def _particle_centre(spec, p):
    """Centre of particle p in the reference's numbering (zone order)."""
    for z in spec.zones:
        if z.is_wall:
            continue
        if p < len(z.sites):
            return z.sites[p][0]
        p -= len(z.sites)
    raise IndexError(p)


def compressive_force_bc():
    """compressive_small with force boundary conditions on four particles,
    one set per time function of ParticleFLoading (particleFLoading.cpp:85-173):
    linear, sin (with a hat_x spatial factor), linear_step and
    linear_slow_fast (with a sin_y spatial factor).  Force densities reach
    ~2e8 N/m^3 by the end of the run (accelerations ~1e5 m/s^2)."""
    s = compressive_small()
    T = s.dt * s.nt
    fmax = 2.0e8
    s.fbc = [
        scene.BCSpec(particles=[0], directions=[1, 2], time_fn="linear", time_params=[fmax / T]),
        scene.BCSpec(particles=[1], directions=[2], time_fn="sin", time_params=[fmax, 1.0 / T],
                     spatial_fn="hat_x", spatial_params=[1.0]),
        scene.BCSpec(particles=[3], directions=[1], time_fn="linear_step",
                     time_params=[fmax / T, 0.25 * T, 0.25 * T]),
        scene.BCSpec(particles=[4, 5], directions=[2], time_fn="linear_slow_fast",
                     time_params=[fmax / T / 500.0, 0.5 * T, 0.5, 1.0],
                     spatial_fn="sin_y", spatial_params=[500.0]),
    ]
    return s


def compressive_displacement_fns():
    """compressive_small with displacement boundary conditions on five
    particles, one per time function of ParticleULoading
    (particleULoading.cpp:115-230) and with the spatial factors: quadratic
    with linear_x, sin with sin_x, rotation about the particle's centre,
    linear with hat_x, constant with linear_y."""
    s = compressive_small()
    T = s.dt * s.nt
    c2 = _particle_centre(s, 2)
    s.ubc = s.ubc + [
        scene.BCSpec(particles=[0], directions=[1], time_fn="quadratic", time_params=[0.05, 2.0e4],
                     spatial_fn="linear_x", spatial_params=[100.0]),
        scene.BCSpec(particles=[1], directions=[2], time_fn="sin", time_params=[1.0e-6, 2.0 / T],
                     spatial_fn="sin_x", spatial_params=[100.0]),
        scene.BCSpec(particles=[2], directions=[1, 2], time_fn="rotation",
                     time_params=[100.0, c2[0], c2[1], 0.0]),
        scene.BCSpec(particles=[3], directions=[2], time_fn="linear", time_params=[1.0],
                     spatial_fn="hat_x", spatial_params=[-0.5]),
        scene.BCSpec(particles=[4], directions=[1, 2], time_fn="constant", time_params=[1.0e-7],
                     spatial_fn="linear_y", spatial_params=[100.0]),
    ]
    return s


def two_particle_const_influence():
    """RNP bonds with the constant influence function (influenceFn.cpp:13-40)."""
    s = two_particle_rnp()
    for z in s.zones:
        z.material.influence_type = 0
    return s


def two_particle_gauss_state():
    """PD state with the Gaussian influence function (influenceFn.cpp:87-122)."""
    s = two_particle_state()
    for z in s.zones:
        z.material.influence_type = 2
    return s


def two_particle_pdelastic_gauss():
    """PD elastic bonds (never break) with the Gaussian influence function."""
    s = scene.two_particle(h_div=8, radius=R, material="PDElasticBond", v0=-1.0, gap=0.02 * R / 8,
                           nt=200)
    for z in s.zones:
        z.material.influence_type = 2
    return s


CASES = {
    "two_particle_rnp": (two_particle_rnp, 400, [1, 2, 10, 41, 100, 200, 400]),
    "two_particle_pmb_impact": (two_particle_pmb_impact, 300, [1, 10, 50, 100, 300]),
    "two_particle_state": (two_particle_state, 300, [1, 10, 100, 300]),
    "two_particle_verlet": (two_particle_verlet, 200, [1, 10, 200]),
    "compressive_small": (compressive_small, 400, [1, 10, 40, 100, 200, 400]),
    "column_3d_small": (column_3d_small, 200, [1, 10, 100, 200]),
    "compressive_force_bc": (compressive_force_bc, 400, [1, 10, 100, 200, 400]),
    "compressive_displacement_fns": (compressive_displacement_fns, 400, [1, 10, 100, 200, 400]),
    "two_particle_const_influence": (two_particle_const_influence, 300, [1, 10, 100, 300]),
    "two_particle_gauss_state": (two_particle_gauss_state, 300, [1, 10, 100, 300]),
    "two_particle_pdelastic_gauss": (two_particle_pdelastic_gauss, 200, [1, 10, 100, 200]),
}
