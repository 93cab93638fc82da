"""Case-file formats: write/read round trips and the structured numbering convention."""
import numpy as np

from tnsgpu import cases, formats


def test_grid_bc_roundtrip(tmp_path):
    m = cases.ramp_mesh(12, 6)
    g, b = tmp_path / "grid.in", tmp_path / "bc.in"
    formats.write_grid_bc(str(g), str(b), m)
    r = formats.read_grid_bc(str(g), str(b))
    assert np.array_equal(r.x, m.x) and np.array_equal(r.y, m.y)  # mm values round-trip exactly
    for k in ("nod", "nc", "nparent", "nghost", "ntype", "nside"):
        assert np.array_equal(getattr(r, k), getattr(m, k)), k


def test_flow_restart_roundtrip(tmp_path):
    f = cases.ramp_flow(2000)
    formats.write_flow(str(tmp_path / "flow.in"), f)
    r = formats.read_flow(str(tmp_path / "flow.in"))
    for k in ("gama", "amol", "local", "niter", "istart", "cfl", "p0", "t0", "pamb", "rtred",
              "npseudo", "iaxis"):
        assert getattr(r, k) == getattr(f, k), k
    c, ri = cases.noisy_restart_state(f, 77)
    formats.write_restart(str(tmp_path / "restart.in"), c, f.rtred, f.npseudo, ri, 123)
    c2, rtred, npseudo, ri2, nold = formats.read_restart(str(tmp_path / "restart.in"), 77)
    assert np.array_equal(c, c2) and rtred == f.rtred and npseudo == 1 and ri2 == ri and nold == 123


def test_structured_numbering_matches_reference_convention():
    # cell (i,j) = i*NJ+j+1 with nodes (i,j),(i+1,j),(i+1,j+1),(i,j+1); ghosts in cell order,
    # sides ascending within a cell (the order of the reference's example bc.in)
    m = cases.nozzle_2d_mesh(5, 3)
    ni, nj = m.shape
    assert m.nod[0].tolist() == [1, nj + 2, nj + 3, 2]
    assert m.nc[0, 1] == nj + 1 and m.nc[0, 2] == 2
    assert m.nparent[:3].tolist() == [1, 1, 2] and m.nside[:3].tolist() == [1, 4, 4]
    assert m.nghosts == 2 * (ni + nj)
    # every boundary face has exactly the ghost of its bc.in line
    for L in range(m.nghosts):
        assert m.nc[m.nparent[L] - 1, m.nside[L] - 1] == m.nghost[L]
    assert set(m.ntype[m.nside == 1]) == {4} and set(m.ntype[m.nside == 3]) == {5}


def test_ramp_first_cell_height():
    m = cases.ramp_mesh(192, 64)
    ni, nj = m.shape
    y = m.y.reshape(ni + 1, nj + 1)
    assert abs((y[0, 1] - y[0, 0]) - 1.0e-5) < 1e-9


def test_renumbered_mesh_is_the_same_mesh():
    """cases.renumbered_mesh shuffles cell and node ids and rotates each cell's faces:
    every cell keeps its corner coordinates in cyclic order, every face still meets the
    neighbour (or ghost) it met before, and each ghost keeps its parent face."""
    m = cases.port_mesh(24, 10)
    g, perm = cases.renumbered_mesh(m, seed=5)
    ne = m.neles
    assert g.neles == ne and g.nods == m.nods and g.nghosts == m.nghosts
    for c in range(ne):
        k = perm[c]
        old = [(m.x[n - 1], m.y[n - 1]) for n in m.nod[c]]
        new = [(g.x[n - 1], g.y[n - 1]) for n in g.nod[k]]
        r = old.index(new[0])
        assert new == old[r:] + old[:r]
        for f in range(4):  # face f of the new cell is face (f + r) % 4 of the old one
            v_old, v_new = m.nc[c, (f + r) % 4], g.nc[k, f]
            assert v_new == (perm[v_old - 1] + 1 if v_old <= ne else v_old)
    for L in range(m.nghosts):
        p_new, s_new = g.nparent[L] - 1, g.nside[L] - 1
        assert g.nc[p_new, s_new] == m.nghost[L]
