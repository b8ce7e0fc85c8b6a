"""VTK frames in the reference's format (include/init.hpp:159-254).

CPU: a numpy restatement of the writer is byte-identical to the reference's
own writer (compiled from source) on random fields.  GPU: hv_write_vtk, which
transposes and byte-swaps on the device, is byte-identical to it on the
fields of a running context, in double and float."""
from __future__ import annotations

import numpy as np
import pytest

from hv_oracle import Reference, reference_available


def vtk_bytes(world, Fx, Fy, Fz, rho, U, dtype):
    """Restatement of output_vtk_header_start / output_vector_field /
    output_scalar_field (include/init.hpp:159-254), frame order of
    src/hyper_vlasov.cpp:79-82."""
    n, dm = world
    nx, ny, nz = n
    G = nx * ny * nz
    d = [dtype(v) for v in dm]
    hdr = ("# vtk DataFile Version 3.0\nVolumetric data\nBINARY\nDATASET STRUCTURED_POINTS\n"
           f"DIMENSIONS {nx} {ny} {nz}\n"
           f"ORIGIN {float(-d[0]):f} {float(-d[1]):f} {float(-d[2]):f}\n"
           f"SPACING {2.0 * float(d[0]) / nx:f} {2.0 * float(d[1]) / ny:f} {2.0 * float(d[2]) / nz:f}\n"
           f"POINT_DATA {G}\n").encode()

    def xfast(a):  # field index (i ny + j) nz + k -> write index (k ny + j) nx + i
        return np.ascontiguousarray(a.reshape(nx, ny, nz).transpose(2, 1, 0)).ravel()

    out = [hdr]
    for s, tag in ((0, "p"), (1, "n")):
        v = np.stack([xfast(F[s * G:(s + 1) * G]) for F in (Fx, Fy, Fz)], axis=1).ravel()
        out.append(f"VECTORS forces_{tag} float\n".encode())
        out.append(v.astype(">f4").tobytes())
    for name, fld in (("density", rho), ("potentials", U)):
        p, q = fld[:G], fld[G:]
        for tag, arr in (("p", p), ("n", q), ("t", (p + q).astype(fld.dtype))):
            out.append(f"SCALARS {name}_{tag} float 1\nLOOKUP_TABLE default\n".encode())
            out.append(xfast(arr).astype(">f4").tobytes())
    return b"".join(out)


@pytest.mark.skipif(not reference_available(), reason="reference harness not built")
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_restated_writer_matches_reference_writer(tmp_path, dtype):
    rng = np.random.default_rng(5)
    world = ((6, 5, 7), (3.0, 2.5, 3.7))
    G = 6 * 5 * 7
    fields = [rng.standard_normal(2 * G).astype(dtype) for _ in range(5)]
    path = tmp_path / "ref.vtk"
    assert Reference(dtype).write_vtk(path, world, *fields) == 0
    assert path.read_bytes() == vtk_bytes(world, *fields, dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_device_writer_matches_reference_format(hv, tmp_path, prec):
    w = hv.CA40_SMALL
    dtype = np.float64 if prec == "f64" else np.float32
    p = hv.workload_particles(w, dtype)
    with hv.Session.from_workload(w, hv.HV_F64 if prec == "f64" else hv.HV_F32) as s:
        s.upload_particles(*p)
        s.initial_solve()
        s.run(2, hv.HV_PATH_FUSED)
        path = tmp_path / "gpu.vtk"
        s.write_vtk(path)
        F = [s.download_field(f) for f in (4, 5, 6)]
        rho, U = s.download_field(1), s.download_field(2)
    assert path.read_bytes() == vtk_bytes(w.world_tuple(), *F, rho, U, dtype)
