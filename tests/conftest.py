import gzip
import shutil
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(ROOT))

QM_FE = 2 * 1.60217733e-19 / (55.845 * 1.660538782e-27)

# small tip used by the device parity tests (about 9k nodes)
SMALL_TIP = dict(cap_radius=1.5e-9, shank_length=2.0e-9, half_angle_deg=0.0, fine_shell=0.6e-9,
                 box_half_width=10e-9, box_height=40e-9, seed=7)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden_dump(tmp_path_factory):
    """The reference's TAPSIM dump of the golden tip (its TetGen mesh and float couplings)."""
    d = tmp_path_factory.mktemp("golden") / "ref_mesh.dump"
    with gzip.open(GOLDEN / "ref_mesh.dump.gz") as f, open(d, "wb") as g:
        shutil.copyfileobj(f, g)
    return d


@pytest.fixture(scope="session")
def ref_events():
    return np.loadtxt(GOLDEN / "ref_events.txt")


@pytest.fixture(scope="session")
def ref_phi0():
    return np.fromfile(GOLDEN / "ref_phi0.bin", np.float32)


@pytest.fixture(scope="session")
def ref_mesh(golden_dump):
    from tapsim_modified_b200.tapsim import Mesh
    return Mesh.from_dump(str(golden_dump), str(GOLDEN / "tip.cfg"))


@pytest.fixture(scope="session")
def small_mesh():
    from tapsim_modified_b200.tapsim import Mesh
    return Mesh.from_tip(**SMALL_TIP)


def free_mask(arrays):
    types = arrays["types"]
    return np.array([not types[int(t)]["dirichlet"] for t in arrays["type"]])


def path_deviation(times, xyz, ref_points, time_scale):
    """Largest distance between a flight path (times [s], positions [m])
    and the in-mesh points of a reference trajectory read from a LogTrajectory
    file (times there are multiplied by the event's time scale), the path
    interpolated linearly at the reference's times; and the reference path's
    largest displacement from its start, to scale it by."""
    rt = ref_points["time"].astype(np.float64) / float(np.float32(time_scale))
    inside = ref_points["tet"] >= 0
    rp = ref_points["position"][inside].astype(np.float64)
    ip = np.stack([np.interp(rt[inside], times, xyz[:, c]) for c in range(3)], axis=1)
    dev = np.linalg.norm(ip - rp, axis=1).max()
    disp = np.linalg.norm(rp - rp[0], axis=1).max()
    return dev, disp


@pytest.fixture(scope="session")
def snapshot_files(tmp_path_factory):
    """The reference's grid and surface snapshots after the first event with
    Fe's permittivity 5 (tests/golden/ref_{grid,surf}_*.00000001.gz),
    unpacked: {name: path}."""
    d = tmp_path_factory.mktemp("snapshots")
    out = {}
    for name in ("ref_grid_ascii", "ref_grid_bin", "ref_surf_ascii", "ref_surf_bin"):
        with gzip.open(GOLDEN / f"{name}.00000001.gz") as f, open(d / name, "wb") as g:
            shutil.copyfileobj(f, g)
        out[name] = str(d / name)
    return out


@pytest.fixture(scope="session")
def ref_mesh_eps5(golden_dump):
    """The golden dump under tip_eps5.cfg (Fe permittivity 5)."""
    from tapsim_modified_b200.tapsim import Mesh
    return Mesh.from_dump(str(golden_dump), str(GOLDEN / "tip_eps5.cfg"))
