"""The reference's GridBlock unit tests (tests/core/test_grid.cpp:39-96 of
GRANITE) on this package's GridBlock, whose flat buffer is the layout the C ABI
takes: cell counts, spacing, coordinates, data access, zero initialisation,
sizes, interior range and the raw field pointer, plus the flat index of
grid.hpp:109-116. (Ranks, neighbour ids and boundary packing belong to the
reference's MPI decomposition, not to this path.)"""
import numpy as np
import pytest

from granite_b200 import GridBlock


@pytest.fixture
def grid():
    return GridBlock(0, 0, (16, 16, 16), (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0), 4, 5)


def test_construction_cell_counts(grid):
    assert [grid.totalCells(d) for d in range(3)] == [24, 24, 24]


def test_cell_spacing(grid):
    for d in range(3):
        assert abs(grid.dx(d) - 2.0 / 16) <= 1e-14


def test_coordinate_mapping(grid):
    assert abs(grid.x(0, 4) - (-1.0 + 0.5 * grid.dx(0))) <= 1e-14
    assert abs(grid.x(0, 4 + 16 - 1) - (1.0 - 0.5 * grid.dx(0))) <= 1e-14


def test_data_access_symmetry(grid):
    grid.set(2, 5, 6, 7, 3.14159)
    assert grid.data(2, 5, 6, 7) == 3.14159


def test_initialized_to_zero(grid):
    assert not np.any(grid.flatBuffer())


def test_total_size_and_interior_range(grid):
    assert grid.totalSize() == 24 * 24 * 24
    assert grid.istart() == 4 and [grid.iend(d) for d in range(3)] == [20, 20, 20]


def test_raw_data_pointer(grid):
    p = grid.rawData(0)
    p[0] = 42.0
    assert grid.data(0, 0, 0, 0) == 42.0
    grid.rawData(3)[7] = 1.5
    assert grid.data(3, 7, 0, 0) == 1.5


def test_flat_index_is_the_reference_layout():
    g = GridBlock(1, 2, (5, 7, 6), (0.0, -1.0, 2.0), (1.0, 1.0, 3.5), 4, 22)
    nx, ny, nz = (g.totalCells(d) for d in range(3))
    stride = nx * ny * nz
    flat = g.flatBuffer()
    flat[:] = np.arange(flat.size, dtype=np.float64)
    for v, i, j, k in [(0, 0, 0, 0), (21, nx - 1, ny - 1, nz - 1), (7, 3, 9, 11), (13, 12, 2, 5)]:
        assert g.data(v, i, j, k) == float(v * stride + i + nx * (j + ny * k))
    assert g.getId() == 1 and g.getLevel() == 2 and g.getNumGhost() == 4 and g.getNumVars() == 22
    assert g.numCells() == (5, 7, 6) and g.lowerCorner() == (0.0, -1.0, 2.0) and g.upperCorner() == (1.0, 1.0, 3.5)
