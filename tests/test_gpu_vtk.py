"""mg_ch_write_vtk (legacy VTK formatted on the GPU) against the host writer
mg_vtk_write, whose "%.3f" lines are byte-identical to the reference's
SfieldFD::writeVTKFile: the files must be equal byte for byte."""
import math

import numpy as np
import pytest

import mesobasic_b200 as mb

pytestmark = pytest.mark.gpu

# exact binary ties at the third decimal, near-ties, signed zeros, tiny
# negatives, large values, non-finite values
SPECIAL = [0.0, -0.0, 0.0625, -0.0625, 0.1875, -0.1875, 2.5, -2.5, 0.0005, -0.0005, 1.0005, 0.9995, -0.9995,
           1e-7, -1e-7, -4e-4, 4e-4, 123456.789, 999.9995, 3.14159265, 1234567890.1235, -987654321.0625,
           3.9e12, -3.9e12, math.nan, -math.nan, math.inf, -math.inf, 0.00049999999999999999, 1.5e-3, 2.5e-3]


def both(tmp_path, sim, field_dims, skips, name):
    dev = tmp_path / f"{name}_dev.vtk"
    host = tmp_path / f"{name}_host.vtk"
    sim.write_vtk(dev, "c", *skips)
    mb.vtk_write(host, "c", sim.get_field(), field_dims, *skips)
    return dev.read_bytes(), host.read_bytes()


@pytest.mark.parametrize("skips", [(1, 1, 1), (2, 1, 1), (3, 2, 2), (40, 1, 1)])
def test_special_values_fp64(tmp_path, skips):
    dims = (16, 5, 3)
    n = int(np.prod(dims))
    vals = np.array((SPECIAL * (n // len(SPECIAL) + 1))[:n], dtype=np.float64)
    vals[-5:] = -vals[-5:]  # more negative non-finite / signed cases
    with mb.CHSim(mb.make_params(*dims, 0.001)) as sim:
        sim.set_field(vals.reshape(dims[::-1]))
        dev, host = both(tmp_path, sim, dims, skips, "special")
    assert dev == host


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
@pytest.mark.parametrize("dims", [(64, 24, 16), (96, 40, 1)])
def test_stepped_field(tmp_path, prec, dims):
    ic = mb.ic_generate(dims, 0.05, 0.4, False, 3)
    with mb.CHSim(mb.make_params(*dims, 0.005, precision=prec)) as sim:
        sim.set_field(ic)
        sim.step(7)
        for skips in [(1, 1, 1), (2, 3, 1)]:
            dev, host = both(tmp_path, sim, dims, skips, f"{prec}_{skips[0]}")
            assert dev == host


def test_two_chunks_and_append(tmp_path):
    dims = (256, 256, 160)  # 10.5 M values: more than one formatting chunk
    ic = mb.ic_generate(dims, 0.0, 0.6, False, 11)
    with mb.CHSim(mb.make_params(*dims, 0.005, precision="fp32")) as sim:
        sim.set_field(ic)
        sim.step(2)
        dev = tmp_path / "big_dev.vtk"
        host = tmp_path / "big_host.vtk"
        for _ in range(2):  # appends, like the reference's ios::app
            sim.write_vtk(dev)
        f = sim.get_field()
        mb.vtk_write(host, "c", f, dims)
        mb.vtk_write(host, "c", f, dims)
    assert dev.read_bytes() == host.read_bytes()


def test_out_of_range_value_is_refused(tmp_path):
    dims = (8, 4, 2)
    vals = np.zeros(dims[::-1])
    vals[1, 2, 3] = 5e12
    with mb.CHSim(mb.make_params(*dims, 0.001)) as sim:
        sim.set_field(vals)
        with pytest.raises(mb.MGError) as e:
            sim.write_vtk(tmp_path / "x.vtk")
    assert "cannot be formatted on the device" in str(e.value)
