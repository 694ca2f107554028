"""The configurations' geometries as the workloads and the bench build them,
without a GPU: config 1 (256^3 @0.5 mm, 360 views, 384^2 @0.8 mm, 40
ellipsoids), config 3 (128^3 @0.9 mm, 180 views, 192^2 @1.2 mm) and the
config-2 tomosynthesis slab (512 x 384 x 64 @0.1/0.1/1.0 mm, 25 views,
1024 x 768 @0.1 mm), and their reduced forms at the same physical extent."""
import math

import pytest

from ct2b200 import diagnostic, differentiable, tomosynthesis


def _extent(vol):
    g = vol.grid
    return tuple(g[i] * g[6 + i] for i in range(3)), tuple(g[3:6])


@pytest.mark.parametrize("scale", [1, 2, 4])
def test_config1_geometry(scale):
    vol, scan, ells = diagnostic.geometry(scale)
    n = 256 // scale
    assert tuple(vol.grid[6:9]) == (n, n, n)
    assert (scan.ns, scan.nu, scan.nv) == (360 // scale, 384 // scale, 384 // scale)
    assert math.isclose(scan.du, 0.8 * scale) and math.isclose(scan.dv, 0.8 * scale)
    size, origin = _extent(vol)
    assert all(math.isclose(s, 128.0) for s in size) and origin == (-64.0, -64.0, -64.0)
    assert len(ells) == 40


@pytest.mark.parametrize("scale", [1, 2, 4])
def test_config3_geometry(scale):
    vol, scan = differentiable.geometry(scale)
    n = 128 // scale
    assert tuple(vol.grid[6:9]) == (n, n, n)
    assert (scan.ns, scan.nu, scan.nv) == (180 // scale, 192 // scale, 192 // scale)
    assert math.isclose(scan.du, 1.2 * scale)
    size, _ = _extent(vol)
    assert all(math.isclose(s, 115.2) for s in size)
    assert differentiable.BATCH == 8 and differentiable.STEPS == 50


@pytest.mark.parametrize("scale", [1, 2, 4])
def test_tomosynthesis_slab(scale):
    vol, scan = tomosynthesis.slab(scale)
    assert tuple(vol.grid[6:9]) == (512 // scale, 384 // scale, 64 // scale)
    assert (scan.ns, scan.nu, scan.nv) == (25, 1024 // scale, 768 // scale)
    assert math.isclose(scan.du, 0.1 * scale)
    size, origin = _extent(vol)
    assert [round(s, 6) for s in size] == [51.2, 38.4, 64.0]
    assert origin == (-25.6, -19.2, -32.0)
