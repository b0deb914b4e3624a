"""Shared 3D CFS-PML case and helpers: a small seeded 3D shot with CFS-PML slabs, its model as the
session builds it, and the oracle mesh made from that model."""
import numpy as np

from cases import case3d


def cpml_case(absorber=1, **kw):
    # 28 x 24 x 26 nodes, h = 10 m, 6/5/6-cell slabs, a force 6 nodes deep, a line of receivers
    c = case3d(nx=28, ny=24, nz=26, relief=6, wavelength=120, duration=0.25, maxSteps=60, sourceX=14, sourceY=12,
               sourceZ=6, absorbing=1, absorbingCells=[6, 5, 6], receiverArray=[1, 2, 12, 0, 24, 1, 1, 1])
    c.update(absorber=absorber, **kw)
    return c


def mesh_from_session(S, sim, params):
    """Oracle/engine mesh dict of a 3D session's own model arrays."""
    info = sim.info()
    m = {k: sim.model(k) for k in ("metrics", "normals", "jacobian", "source", "damping")}
    for k in ("materialLambda", "materialMu", "materialDensity", "sourceGradient0", "sourceGradient1", "sourceGradient2"):
        v = sim.model(k)
        if v.size:
            m[k] = v
    rates = sim.model("gslsRates")
    if rates.size:  # GSLS: mechanisms, rates and strengths
        m["mechanisms"], m["rates"] = int(rates.size), rates.tolist()
        for l in range(rates.size):
            m[f"deltaP{l}"], m[f"deltaS{l}"] = sim.model(f"deltaP{l}"), sim.model(f"deltaS{l}")
    shape = sim.model("cpmlShape")
    if shape.size and shape[3] > 0:
        m.update(cpmlX=sim.model("cpmlX"), cpmlY=sim.model("cpmlY"), cpmlZ=sim.model("cpmlZ"), cpmlWidthX=int(shape[0]),
                 cpmlWidthY=int(shape[1]), cpmlWidthZ=int(shape[2]), cpmlCount=int(shape[3]))
    rho, vp, vs = params.get("density", 2200.0), params.get("vp", 3000.0), params.get("vs", 1700.0)
    m.update(nx=info["nx"], ny=info["ny"], nz=info["nz"], h=info["h"], dt=info["dt"], density=rho,
             mu=rho * vs * vs, frequency=params.get("frequency", 12.0))
    m["lambda"] = rho * (vp * vp - 2.0 * vs * vs)
    kind = int(params.get("sourceKind", 0))
    m["sourceAmplitude"] = params.get("sourceMoment", 2e9) if kind else params.get("sourceForce", 2e8)
    d = np.asarray(params.get("sourceDirection", (0, 0, 1)), dtype=np.float64)
    m["sourceDirection"] = (0.0, 0.0, 0.0) if kind else tuple(d / np.linalg.norm(d))
    return m


def receiver_nodes(S, sim):
    """Padded node indices of the session's receivers (the line at depth 0 of cpml_case)."""
    info = sim.info()
    nx, ny = info["nx"], info["ny"]
    return np.array([(2 + r + 3) + nx * ((12 + 3) + ny * 3) for r in range(info["receivers"])], dtype=np.int64)
