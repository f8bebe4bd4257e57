"""The oracle's slab entries (marching cubes and PLIC over the cell layers k0..k1-1 of a full grid)
must reproduce the whole-grid oracle's layers bit for bit: they are what the large-grid device
parity tests compare against, so a slab may not re-base its coordinates or lose a neighbour."""
import numpy as np
import pytest

from helpers import cc, po, assert_cells_bitwise, bits


def _slab_of(cols, lay, k0, k1):
    return {k: v[lay * k0:lay * k1] for k, v in cols.items()}


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_mc_slab_equals_whole_grid_layers(prec):
    g = cc.CartesianGrid((-1.1, -0.95, -1.05), (24, 21, 19), (0.09, 0.1, 0.11))
    tape = cc.flatten(cc.workloads.csg_body(3), 3)
    table = cc.mc_tables.project_table()
    phi, ref = po.mc_update(g, tape, table, prec)
    lay, nlay = g.n[0] * g.n[1], (g.n[0] + 1) * (g.n[1] + 1)
    for k0, k1 in ((0, 4), (7, 12), (15, 19), (0, 19)):
        sphi, got = po.mc_update_slab(g, tape, table, prec, k0, k1)
        assert np.array_equal(bits(sphi), bits(phi[nlay * k0:nlay * (k1 + 1)]))
        assert_cells_bitwise(got, _slab_of(ref, lay, k0, k1), label=f"slab {k0}..{k1}")
    assert (ref["kind"] == 2).sum() > 200


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_plic_slab_equals_whole_grid_layers(prec):
    g = cc.workloads.unit_grid(20)
    tape = cc.flatten(cc.workloads.sphere_cloud(1, 12), 3)
    cols, nrm, icp, val = po.plic_update(g, tape, prec)
    lay = g.n[0] * g.n[1]
    for k0, k1 in ((0, 3), (8, 13), (17, 20)):
        c2, n2, i2, v2 = po.plic_update_slab(g, tape, prec, k0, k1)
        sl = slice(lay * k0, lay * k1)
        assert np.array_equal(bits(n2), bits(nrm[sl])) and np.array_equal(bits(i2), bits(icp[sl]))
        assert np.array_equal(v2, val[sl])
        assert_cells_bitwise(c2, _slab_of(cols, lay, k0, k1), fields=("kind", "volume_fraction", "face_fraction"),
                             label=f"plic slab {k0}..{k1}")
    assert (cols["kind"] == 2).sum() > 100


def test_slab_rejects_bad_ranges():
    g = cc.workloads.csg_grid(8)
    tape = cc.flatten(cc.workloads.csg_body(0), 3)
    with pytest.raises(AssertionError):
        po.mc_update_slab(g, tape, cc.mc_tables.project_table(), 0, 5, 5)
    with pytest.raises(AssertionError):
        po.plic_update_slab(g, tape, 0, 4, 9)
