"""VTK output of device fields: the device encoder (flb_vtk_field_base64)
against the oracle's restatement, and the host classes' vtmo writers against
the reference's own files, byte for byte."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import freelb_b200 as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def fill_fields(lat, n, seed):
    rng = np.random.default_rng(seed)
    rho = (1 + 0.01 * rng.standard_normal(n)).astype(lat.real)
    u = (0.05 * rng.standard_normal((n, 3))).astype(lat.real)
    lat.upload_field("rho", rho)
    lat.upload_field("u", u)
    return rho, u


@pytest.mark.parametrize("storage", ["fp32", "fp16s", "fp64"])
@pytest.mark.parametrize("overlap", [0, 1, 2])
def test_device_body_matches_oracle(gpu_ok, storage, overlap):
    nx, ny, nz = 13, 9, 7
    lat = F.Lattice(nx, ny, nz, 0.6, storage=storage)
    rho, u = fill_fields(lat, nx * ny * nz, 3)
    flags = np.random.default_rng(4).integers(0, 255, nx * ny * nz, dtype=np.uint8)
    lat.upload_flags(flags)
    mesh = (nx, ny, nz)
    assert lat.vtk_body("flag", overlap) == O.vtk_body(O.vtk_crop(flags, mesh, overlap))
    for dt in (np.float32, np.float64):
        want_r = O.vtk_crop(rho, mesh, overlap).astype(dt)
        assert lat.vtk_body("rho", overlap, dtype=dt) == O.vtk_body(want_r)
        want_u = O.vtk_crop(u, mesh, overlap, ncomp=3).astype(dt)
        assert lat.vtk_body("u", overlap, dtype=dt) == O.vtk_body(want_u)
    # unit conversion in the field's type, then the output type
    T = lat.real
    sc, off = 1.7, 0.25
    want = (O.vtk_crop(rho, mesh, overlap) * T(sc) + T(off)).astype(np.float64)
    assert lat.vtk_body("rho", overlap, dtype=np.float64, scale=sc, offset=off) == O.vtk_body(want)
    want = O.vtk_crop(u, mesh, overlap, ncomp=3) * T(sc)
    assert lat.vtk_body("u", overlap, scale=sc) == O.vtk_body(want)


def test_device_body_of_each_block(gpu_ok):
    sizes = [(10, 8, 6), (7, 7, 7), (16, 5, 9)]
    lat = F.Lattice.blocks([(a, b, c, 0, 0, 0, 1.0 / 0.6) for a, b, c in sizes], 0.6,
                           mode="independent")
    for k, (a, b, c) in enumerate(sizes):
        rng = np.random.default_rng(k)
        r = rng.random(a * b * c).astype(np.float32)
        lat.upload_field("rho", r, block=k)
        assert lat.vtk_body("rho", 1, block=k) == O.vtk_body(O.vtk_crop(r, (a, b, c), 1))


@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("overlapth,steps", [(-1, 0), (0, 0), (0, 5)])
def test_host_class_files_equal_reference_files(gpu_ok, precision, overlapth, steps):
    """cavity3d_vtk (host classes, device encoder for rho / velocity and their
    Phys forms) and the reference harness (vtmo writers) write identical .vti
    and .vtm files from the same RHO and VELOCITY fields."""
    from freelb_b200 import build as B
    exe = B.build_example("cavity3d_vtk")
    ref_exe = O.ref_binary(np.float64 if precision == "fp64" else np.float32)
    if ref_exe is None:
        pytest.skip("reference harness not built")
    ni = 9
    n = ni + 2
    rng = np.random.default_rng(11)
    rho = 1 + 0.01 * rng.standard_normal(n ** 3)
    u = 0.05 * rng.standard_normal((n ** 3, 3))
    dt = np.float64 if precision == "fp64" else np.float32
    with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
        f64 = os.path.join(d2, "fields64.bin")
        np.concatenate([rho, u.ravel()]).astype(np.float64).tofile(f64)
        fT = os.path.join(d1, "fieldsT.bin")
        np.concatenate([rho, u.ravel()]).astype(dt).tofile(fT)
        env = dict(os.environ, FLB_VTK_NAME="cav", FLB_VTK_OVERLAP=str(overlapth),
                   FLB_FIELDS_FILE=fT, OMP_NUM_THREADS="1")
        subprocess.run([ref_exe, "bgk", str(ni), "0.6", "0.1", str(steps), "0", "-"], cwd=d1,
                       env=env, check=True, capture_output=True)
        args = [exe, str(ni), "0.6", "0.1", str(steps), str(overlapth), "cav", f64]
        if precision == "fp64":
            args.append("fp64")
        r = subprocess.run(args, cwd=d2, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        for name in (f"cav{steps}.vtm", f"cav_T{steps}_B0.vti"):
            a = open(os.path.join(d2, "vtkoutput", "vtidata", name), "rb").read()
            b = open(os.path.join(d1, "vtkoutput", "vtidata", name), "rb").read()
            assert a == b, name
