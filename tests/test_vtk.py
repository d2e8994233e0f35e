"""VTK output: the reference's vtmo writers (src/io/vtm_writer.h:288-663) run in
the reference harness, the oracle's restatement of their DataArray bodies, and
the C++ host classes' vtmo writers (flag field encoded on the host; the device
encoder is covered by tests/test_vtk_gpu.py)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT
from oracle import oracle as O

needs_ref = pytest.mark.skipif(O.ref_binary(np.float32) is None,
                               reason="reference harness not built here")


def run_ref(d, ni, steps, overlapth, dtype=np.float32, fields=None):
    env = dict(os.environ, FLB_VTK_NAME="cav", FLB_VTK_OVERLAP=str(overlapth), OMP_NUM_THREADS="1")
    if fields is not None:
        f = os.path.join(d, "fields.bin")
        np.concatenate([fields[0].ravel(), fields[1].ravel()]).astype(dtype).tofile(f)
        env["FLB_FIELDS_FILE"] = f
    subprocess.run([O.ref_binary(dtype), "bgk", str(ni), "0.6", "0.1", str(steps), "0", "-"],
                   cwd=d, env=env, check=True, capture_output=True)
    return os.path.join(d, "vtkoutput", "vtidata")


@needs_ref
@pytest.mark.parametrize("overlapth", [-1, 0, 1])
def test_oracle_bodies_match_reference_writer(overlapth):
    """Each DataArray of the reference's .vti decodes to the cropped field and
    re-encodes, through the oracle, to the same characters."""
    ni, n = 6, 8
    rng = np.random.default_rng(5)
    rho = 1 + 0.01 * rng.standard_normal(n ** 3)
    u = 0.05 * rng.standard_normal((n ** 3, 3))
    with tempfile.TemporaryDirectory() as d:
        out = run_ref(d, ni, 0, overlapth, fields=(rho, u))
        arrs = O.vtk_arrays(os.path.join(out, "cav_T0_B0.vti"))
    ov = 1 if overlapth == 0 else 0
    assert set(arrs) == {"flag", "rho", "velocity", "physRho", "physVelocity"}
    fl = O.vtk_crop(O.cavity_flags(ni), (n, n, n), ov)
    assert arrs["flag"][:2] == ("UInt8", 1) and arrs["flag"][2] == O.vtk_body(fl)
    r32 = O.vtk_crop(rho.astype(np.float32), (n, n, n), ov)
    assert arrs["rho"][:2] == ("Float32", 1) and arrs["rho"][2] == O.vtk_body(r32)
    u32 = O.vtk_crop(u.astype(np.float32), (n, n, n), ov, ncomp=3)
    assert arrs["velocity"][:2] == ("Float32", 3) and arrs["velocity"][2] == O.vtk_body(u32)
    assert np.array_equal(O.vtk_decode(arrs["velocity"][2], np.float32), u32)


def test_oracle_body_padding_cases():
    """Sizes 1, 2 and 3 bytes mod 3: '=' padding of both streams."""
    import base64
    for n in range(1, 8):
        data = np.arange(n, dtype=np.uint8)
        body = O.vtk_body(data)
        assert body[:8] == base64.b64encode(np.uint32(n).tobytes()).decode()
        assert O.vtk_decode(body, np.uint8).tolist() == list(range(n))


@needs_ref
@pytest.mark.parametrize("overlapth", [-1, 0])
def test_host_classes_write_the_reference_flag_file(overlapth):
    """vtmo::vtmWriter + vtmo::ScalarWriter of the host classes (flag field,
    encoded on the host) write the reference's .vtm and the reference's .vti
    up to the end of the flag array, byte for byte."""
    from freelb_b200 import build as B
    exe = B.build_example("cavity3d_vtk")
    ni = 7
    with tempfile.TemporaryDirectory() as d1, tempfile.TemporaryDirectory() as d2:
        ref = run_ref(d1, ni, 3, overlapth)
        subprocess.run([exe, str(-ni), "0.6", "0.1", "3", str(overlapth), "cav"], cwd=d2,
                       check=True, capture_output=True)
        ours = os.path.join(d2, "vtkoutput", "vtidata")
        assert open(os.path.join(ours, "cav3.vtm"), "rb").read() == \
            open(os.path.join(ref, "cav3.vtm"), "rb").read()
        a = open(os.path.join(ours, "cav_T3_B0.vti"), "rb").read()
        b = open(os.path.join(ref, "cav_T3_B0.vti"), "rb").read()
        cut = b.index(b"</DataArray>\n") + len(b"</DataArray>\n")
        assert a[:cut] == b[:cut]
        assert a[cut:] == b"</PointData>\n</Piece>\n</ImageData>\n</VTKFile>\n"
