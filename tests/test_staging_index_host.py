"""Host check of the index arithmetic of the staged edge scan (staged_scan in csrc/rak_lpa.cuh),
restated step for step: for ranges of every length and every 4-byte misalignment of the edge
array, each lane must visit exactly its edges eb+lane, eb+lane+32, ... in order; every shared-memory
read must fall inside the tile (offsets 0..STG_TILE-1) and hold a copied edge; every global read must
fall inside [eb, ee); every bulk copy must start and end on 16-byte boundaries inside [eb, ee)."""
import pytest

STG_TILE, B = 256, 4


def walk(eb, ee, base_mis):
    """base_mis: the edge array's address modulo 16, in 4-byte units (0..3)."""
    addr = lambda e: (base_mis + e) * 4
    cs = eb + (((16 - (addr(eb) & 15)) & 15) >> 2)
    cs = min(cs, ee)
    ce = cs + ((ee - cs) & ~3)
    nt = (ee - cs + STG_TILE - 1) // STG_TILE if ee > eb else 0
    if ee > eb and nt < 1:
        nt = 1
    copies = []
    for k in range(nt):
        tb = cs + k * STG_TILE
        te = min(tb + STG_TILE, ce)
        if te > tb:
            copies.append((tb, te))
    visits = {lane: [] for lane in range(32)}
    for lane in range(32):
        rel = eb - cs + lane
        for k in range(nt):
            tb = cs + k * STG_TILE
            whole = k > 0 and tb + STG_TILE <= ce
            if whole:
                assert 0 <= rel < 32
                for b0 in range(0, STG_TILE // 32, B):
                    for j in range(B):
                        x = rel + (b0 + j) * 32
                        assert 0 <= x < STG_TILE and tb + x < ce
                        visits[lane].append(("s", tb + x))
                rel += STG_TILE
            else:
                hi = ee - tb if k + 1 >= nt else STG_TILE
                se = STG_TILE if tb + STG_TILE < ce else ce - tb
                while rel < hi:
                    left = (hi - rel + 31) >> 5
                    take = min(left, B)
                    for j in range(take):
                        x = rel + j * 32
                        if 0 <= x < se:
                            assert x < STG_TILE
                            visits[lane].append(("s", tb + x))
                        else:
                            assert eb <= tb + x < ee
                            visits[lane].append(("g", tb + x))
                    rel += take * 32
            rel -= STG_TILE
    return copies, visits


@pytest.mark.parametrize("mis", [0, 1, 2, 3])
def test_every_edge_once_in_order_and_in_bounds(mis):
    lengths = list(range(0, 70)) + [255, 256, 257, 259, 260, 511, 512, 513, 515, 516, 1023, 1024, 1025, 1027, 1500, 2048, 2051, 4099, 8192]
    for eb in (0, 1, 2, 3, 5, 1000, 1001, 4097):
        for n in lengths:
            ee = eb + n
            copies, visits = walk(eb, ee, mis)
            for tb, te in copies:
                assert eb <= tb < te <= ee
                assert ((mis + tb) * 4) % 16 == 0 and ((te - tb) * 4) % 16 == 0
            for lane in range(32):
                got = [e for _, e in visits[lane]]
                assert got == list(range(eb + lane, ee, 32)), (eb, n, mis, lane)
                for kind, e in visits[lane]:
                    if kind == "s":
                        assert any(tb <= e < te for tb, te in copies)
