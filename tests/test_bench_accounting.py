"""The bench's accounting of algorithmic work (CPU only): the cell-sweeps and bytes of
one V-cycle from the per-routine word counts of the reference's loops, at the
obstacle-flow configuration (256 x 256, ngrid 5, nswpm 2, nswpp 10)."""
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cycle_accounting():
    sys.path.insert(0, REPO)
    import bench
    from mgfvm import configs
    cfg = configs.c1(10.0, seed=1)
    # visits x interior cells: 65536 + 2 (16384 + 4096 + 1024) + 256 = 108800
    visits_cells = 65536 + 2 * (16384 + 4096 + 1024) + 256
    assert bench.cell_sweeps_per_cycle(cfg) == (3 * 2 + 10) * visits_cells == 1_740_800
    # 85 words of assembly + 8 per cell-sweep per cell and visit; 124 words per fine
    # cell of each of the four transfers
    words = visits_cells * (85 + 8 * 16) + (65536 + 16384 + 4096 + 1024) * 124
    assert bench.cycle_bytes(cfg) == 8 * words == 271_738_880
