"""The roofline arithmetic of bench.py on the wave226 workload (768 x 768 x
384 nodes, a 12-node PML on the four side faces and the bottom, a free
surface on top), counted here face by face: 84 B per node-update (v, u read
and written, mr, gam, lam, mu, yy, 1/V, and x, y, z) plus 24 B for each PML
slab a node (p memory) or a cell (g memory) belongs to."""
import bench


def test_wave226_algorithmic_bytes():
    nx, ny, nz = 768, 768, 384
    npml = 12
    nodes = nx * ny * nz
    # node slabs: two x faces, two y faces, the bottom
    pn = npml * (2 * ny * nz + 2 * nx * nz + nx * ny)
    # cell slabs, the same faces over the cells
    cx, cy, cz = nx - 1, ny - 1, nz - 1
    pc = npml * (2 * cy * cz + 2 * cx * cz + cx * cy)
    assert bench.pml_memberships((nx, ny, nz)) == (pn, pc)
    per_node = bench.algorithmic_bytes_per_node((nx, ny, nz))
    assert abs(per_node - (84.0 + 24.0 * (pn + pc) / nodes)) < 1e-9
    assert abs(per_node * nodes - 20042810784.0) < 1.0
    assert 88.4 < per_node < 88.6
