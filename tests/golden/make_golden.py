"""Regenerates the golden fixtures of tests/golden/ from the CPU oracle.

The reference (Julia) cannot run on any machine of this build and its own
tests pin no numerical results, so the fixtures come from the oracle (the
FP64 restatement of the reference's CPU integrator), pinned itself by
tests/test_oracle_physics.py and tests/test_ref_integrator.py. Small cases:
10x10 pixels (flat sphere 16x16, thick disk 8x8), 8 spectral bins, tolerance 1e-8, both step
modes; the per-bin scenes (PERBIN below); the skybox scenes (SKYBOX below).
Run: python tests/golden/make_golden.py (all), or with --skybox (the skybox scenes).
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import oracle as O  # noqa: E402
from rtwca_b200 import abi, configs  # noqa: E402

CASES = {"minkowski_sphere": 16, "schwarzschild_disk": 10, "kerr_thin_disk": 10, "kerr_thick_disk": 8}
N_COLORS = 8

# the per-bin scenes: Powehi ("m87" camera, 12 px wide, 3 bins), Synchro_Test
# ("synch" camera, 16 px wide, 3 bins), both steps, tolerance 1e-6; the
# synchrotron torus (8 x 8, 4 bins, tolerance 1e-8, FSAL only)
PERBIN = {"powehi": ("ref", "fsal"), "synchro_test": ("ref", "fsal"), "synchrotron_torus": ("fsal",)}


# the skybox scenes, with synthetic 8-texel cube maps (the reference's PNGs are
# not in its repository); the oracle side only for now
SKYBOX = {"wormhole_bundles": ("fsal",), "cart_sphere": ("ref", "fsal"), "cart_sphere_bundles": ("fsal",)}


def skybox_case(name):
    """(scene, camera, colours, skyboxes, ray_bundles) of a skybox fixture."""
    rng = np.random.default_rng(12)
    sky = tuple(rng.uniform(0, 1, (24, 32, 3)).astype(np.float32) for _ in range(2))
    col = np.array([467.0, 532.0, 630.0])
    if name == "wormhole_bundles":
        return configs.wormhole_scene(), configs.wormhole_camera(12, 1e-6), col, sky, True
    return (configs.cart_sphere_scene(), configs.cart_sphere_camera(12, 1e-6), col, (sky[0], None),
            name == "cart_sphere_bundles")


def perbin_case(name):
    if name == "powehi":
        return configs.powehi_scene(), configs.powehi_camera(12, 1e-6), np.array([400.0, 550.0, 700.0])
    if name == "synchro_test":
        return configs.synchro_scene(), configs.synchro_camera(16, 1e-6), np.array([400.0, 550.0, 700.0])
    sc, cam, col = configs.torus_problem(x_pix=8, tol=1e-8)
    return sc, cam, col[::8]


def case(name, integrator):
    scene, cam, _ = configs.workload(name, x_pix=CASES[name])
    colors = configs.log_spaced_colors(N_COLORS)
    return scene, cam, colors, integrator


def main():
    O.build()
    for name in CASES:
        for integ, tag in ((abi.DP45_REF_COMPAT, "ref"), (abi.DP45_FSAL, "fsal")):
            scene, cam, colors, _ = case(name, integ)
            res = O.render(scene, cam, colors, integrator=integ)
            np.savez_compressed(HERE / f"{name}_{tag}.npz", colors=colors, xyz=res["xyz"], term_class=res["class"],
                                steps=res["steps"], spectrum=res["spectrum"], tau=res["tau"][:, 0],
                                state=res["state"])
            print(name, tag, np.bincount(res["class"], minlength=7).tolist())
    for name, tags in PERBIN.items():
        for tag in tags:
            integ = abi.DP45_REF_COMPAT if tag == "ref" else abi.DP45_FSAL
            scene, cam, colors = perbin_case(name)
            res = O.render(scene, cam, colors, integrator=integ)
            np.savez_compressed(HERE / f"{name}_{tag}.npz", colors=colors, xyz=res["xyz"], term_class=res["class"],
                                steps=res["steps"], spectrum=res["spectrum"], tau=res["tau"][:, 0],
                                state=res["state"])
            print(name, tag, np.bincount(res["class"], minlength=7).tolist())
    skybox_main()


def skybox_main():
    O.build()
    for name, tags in SKYBOX.items():
        for tag in tags:
            integ = abi.DP45_REF_COMPAT if tag == "ref" else abi.DP45_FSAL
            scene, cam, colors, sky, bundles = skybox_case(name)
            res = O.render(scene, cam, colors, integrator=integ, skybox=sky, ray_bundles=bundles)
            np.savez_compressed(HERE / f"{name}_{tag}.npz", colors=colors, xyz=res["xyz"], term_class=res["class"],
                                steps=res["steps"], spectrum=res["spectrum"], tau=res["tau"][:, 0],
                                state=res["state"])
            print(name, tag, np.bincount(res["class"], minlength=7).tolist())


if __name__ == "__main__":
    skybox_main() if sys.argv[1:] == ["--skybox"] else main()
