"""Reader for the tagged binary dumps written by oracle/ref_driver.cpp.

ORACLE TEST INFRASTRUCTURE ONLY: used by tests to load the reference's own
state; never imported by the product package.
"""
import struct

import numpy as np

_DT = {0: np.float64, 1: np.float32, 2: np.uint8, 3: np.int64}


def read_dump(path):
    """Return {name: ndarray} for one dump file."""
    out = {}
    with open(path, "rb") as fh:
        data = fh.read()
    if data[:8] != b"PDDUMP01":
        raise ValueError(f"{path}: not a PDDUMP01 file")
    p = 8
    while p < len(data):
        (ln,) = struct.unpack_from("<I", data, p)
        p += 4
        name = data[p:p + ln].decode()
        p += ln
        dt, n = struct.unpack_from("<IQ", data, p)
        p += 12
        t = np.dtype(_DT[dt])
        out[name] = np.frombuffer(data, dtype=t, count=n, offset=p).copy()
        p += n * t.itemsize
    return out


def scene_from_dump(d, name="ref"):
    """Build a peridem_b200.model.Scene from a reference init dump: the
    ModelData the reference's DEMModel::init produced, in the reference's
    own neighbour-list order."""
    from peridem_b200.model import Scene, BCSet

    def s(k):
        return d[k][0]

    N = int(s("N"))
    Np = int(s("Np"))
    dim = int(s("dim"))
    mp = d["p_mat_params"].reshape(Np, 8)
    nz = int(s("nzones"))
    sets = {}
    for pre in ("ubc", "fbc"):
        out = []
        for k in range(int(s(pre + "_nsets"))):
            key = f"{pre}_{k}_"
            dirs = d[key + "dirs"]
            mask = 0
            for q in dirs:
                mask |= 1 << (int(q) - 1)
            tp = np.zeros(4)
            tpv = d[key + "time_params"][:4]
            tp[:len(tpv)] = tpv
            sp = np.zeros(2)
            spv = d[key + "spatial_params"][:2]
            sp[:len(spv)] = spv
            tcode = int(s(key + "time"))
            out.append(BCSet(time_fn=tcode if tcode >= 0 else 99, spatial_fn=int(s(key + "spatial")),
                             dir_mask=mask, zero=bool(s(key + "zero")), time_params=tp,
                             spatial_params=sp, particle_sel=d[key + "proc"],
                             node_sel=d[key + "mask"],
                             particle_box=d[key + "box"].reshape(Np, 6)))
        sets[pre] = out
    ic_v = d["ic_v"] if int(s("ic_active")) else None
    return Scene(
        dim=dim, dt=float(s("dt")), nt=int(s("Nt")),
        xref=d["xRef"].reshape(N, 3), vol=d["vol"], fix=d["fix"],
        ptid=d["ptId"].astype(np.uint64),
        p_start=d["p_globStart"], p_end=d["p_globEnd"], p_center=d["p_center"],
        p_type=d["p_type"], p_zone=d["p_zone"], p_compute_force=d["p_computeForce"],
        p_all_fixed=d["p_allDofsConstrained"], p_material=d["p_mat_type"],
        p_horizon=d["p_horizon"], p_h=d["p_h"], p_density=d["p_density"], p_rc=d["p_Rc"],
        p_kn=d["p_Kn"], p_bound_r=d["p_boundR"], p_mat=mp[:, :6],
        inf_type=int(s("inf_type")), inf_params=d["inf_params"],
        gravity=d["gravity"], time_scheme=int(s("time_disc")),
        multi_particle=bool(s("is_multi")), n_zones=nz,
        c_rc=d["c_Rc"], c_kn=d["c_Kn"], c_mu=d["c_mu"], c_betan=d["c_betan"],
        c_kappa=d["c_kappa"], max_contact_r=float(s("maxContactR")),
        search_factor=float(s("sFactor")), search_interval=int(s("neighUpdateInterval")),
        test=int(s("test")), test_wall=int(s("cmp_wall")), test_dir=max(int(s("cmp_dir")), 0),
        test_interval=int(s("dtTestOut")),
        # state right after DEMModel::init, before the integrate() prelude:
        # BaseParticle sets d_x = d_xRef and u = v = 0 (baseParticle.cpp:131-134)
        x=d["xRef"].reshape(N, 3).copy(), u=np.zeros((N, 3)), v=np.zeros((N, 3)),
        mx=d["mX"], pd_rowptr=d["pd_rowptr"].astype(np.uint64),
        pd_col=d["pd_col"].astype(np.uint64), bond_state=None,
        ubc=sets["ubc"], fbc=sets["fbc"], ic_velocity=ic_v,
        ic_particles=d["ic_plist"].astype(np.uint64), name=name)
