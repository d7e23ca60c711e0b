"""Small seeded scenes for parity tests (sizes the reference finishes in
seconds).  Each entry: (scene spec factory, steps, dump steps)."""
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


CASES = {
    "two_particle_rnp": (two_particle_rnp, 400, [1, 2, 10, 41, 100, 200, 400]),
    "two_particle_pmb_impact": (two_particle_pmb_impact, 300, [1, 10, 50, 100, 300]),
    "two_particle_state": (two_particle_state, 300, [1, 10, 100, 300]),
    "two_particle_verlet": (two_particle_verlet, 200, [1, 10, 200]),
    "compressive_small": (compressive_small, 400, [1, 10, 40, 100, 200, 400]),
    "column_3d_small": (column_3d_small, 200, [1, 10, 100, 200]),
}
