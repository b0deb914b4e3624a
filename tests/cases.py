"""Small seeded parity cases in the reference's parameter vocabulary.

2D keys follow Seis2D::Curvilinear::Parameters (include/Seis2D/CurvilinearSolver2D.hpp:29-57),
3D keys follow Seis3D::Curvilinear::SimulationParameters (include/Seis3D/CurvilinearSolver.hpp:70-95);
layer rows are (thickness, vp, vs, density[, qp, qs]).  They cover the branches of the step:
sponge and external/internal CFS-PML, force and moment sources, flat and curved surfaces,
GSLS with 1 and 3 mechanisms, surface and buried sources, layered materials.
"""

LAYERS2 = [20, 1500, 700, 2050, 100, 60, 50, 2500, 1300, 2250, 100, 60, 0, 4000, 2300, 2650, 100, 60]


def case2d(**kw):
    c = dict(nx=40, nz=30, spacing=5, relief=3, wavelength=100, frequency=20, duration=0.05, maxSteps=40,
             sourceX=20, sourceZ=8, receiverStart=2, receiverCount=10, receiverStride=3, receiverDepth=0)
    c.update(kw)
    return c


CASES_2D = {
    "sponge_force": case2d(absorber=0, spongeX=6, spongeZ=6),
    "cpml_external_moment_layers": case2d(absorber=1, spongeX=6, spongeZ=6, externalAbsorption=1, sourceKind=1,
                                          layered=1, layers=LAYERS2),
    "gsls3_cpml_surface_force": case2d(absorber=1, spongeX=6, spongeZ=6, attenuation=1, mechanisms=3,
                                       qMinFrequency=5, qMaxFrequency=60, qReferenceFrequency=25, qp=60, qs=30,
                                       sourceZ=0, sourceDirection=[0.3, 0, 1]),
    "gsls1_layers_sponge": case2d(absorber=0, spongeX=5, spongeZ=5, attenuation=1, mechanisms=1, layered=1,
                                  layers=[30, 1200, 600, 1900, 40, 20, 0, 2600, 1400, 2200, 120, 60]),
    "flat_surface_force": case2d(relief=0, absorber=0, sourceZ=0, receiverDepth=1),
    "cpml_internal_steep": case2d(nx=48, nz=36, relief=6, wavelength=60, absorber=1, spongeX=7, spongeZ=5,
                                  sourceX=24, sourceZ=10, sourceKind=1, receiverStart=8, receiverCount=8,
                                  receiverStride=4),
}


def case3d(**kw):
    c = dict(nx=16, ny=14, nz=16, spacing=10, relief=8, wavelength=80, frequency=12, duration=0.1, maxSteps=16,
             sourceX=8, sourceY=7, sourceZ=5, absorbingCells=[3, 3, 3], receiverArray=[3, 2, 2, 0, 5, 3, 2, 2])
    c.update(kw)
    return c


CASES_3D = {
    "force": case3d(),
    "moment_layered": case3d(sourceKind=1, layered=1, layerDepthMode=1,
                             layers=[30, 1200, 600, 1800, 40, 2400, 1300, 2100, 0, 3800, 2200, 2400]),
    "flat_tilted_force": case3d(relief=0, sourceZ=2, sourceDirection=[0.2, 0.1, 1]),
}
