"""The per-cell cap rule of the warp-per-body pair search equals the
reference's sequential loop.

findPairsInCell (G3/bt3dGridBroadphaseOCL.cl:129-131, 159-162) appends a
body's candidates cell by cell and stops a cell at the first candidate past
curr_max = maxPairsPerBody - 1, counting one overflow; a cell scanned to its
bucket cap while its bucket holds more bodies counts one cell overflow. The
warp form computes every cell's count independently and derives the kept
pairs and both overflow counts from an exclusive scan of the counts
(k_find_pairs_warp). Both rules are restated here in plain Python and
compared on random cell contents, bucket caps, pair caps and large-body
lists (the large-body pass in 32-wide chunks, as the warp form's ballots).
"""
import random


def sequential(cells, large, cap, bucket_cap):
    cnt, out, ovf, covf = 0, [], 0, 0
    for cell in cells:
        if cell is None:
            continue
        entries, longer = cell
        full = False
        for is_cand, other in entries[:bucket_cap]:
            if is_cand:
                if cnt >= cap:
                    ovf += 1
                    full = True
                    break
                out.append(other)
                cnt += 1
        if not full and longer:
            covf += 1
    for hit, body in large:
        if hit:
            if cnt >= cap:
                ovf += 1
                break
            out.append(body)
            cnt += 1
    return out, ovf, covf


def per_cell(cells, large, cap, bucket_cap):
    counts = [0 if c is None else sum(1 for is_cand, _ in c[0][:bucket_cap] if is_cand) for c in cells]
    out = [None] * cap
    ovf = covf = 0
    before_all = 0
    for cell, c in zip(cells, counts):
        before = min(before_all, cap)
        room = cap - before
        keep = min(c, room)
        cell_ovf = c > room
        ovf += int(cell_ovf)
        if cell is not None and not cell_ovf and cell[1]:
            covf += 1
        kept = [o for is_cand, o in cell[0][:bucket_cap] if is_cand][:keep] if keep > 0 else []
        for k, o in enumerate(kept):
            out[before + k] = o
        before_all += c
    cnt = min(before_all, cap)
    for l0 in range(0, len(large), 32):
        hits = [body for hit, body in large[l0:l0 + 32] if hit]
        for rank, body in enumerate(hits):
            if cnt + rank < cap:
                out[cnt + rank] = body
        if cnt + len(hits) > cap:
            ovf += 1
            cnt = cap
            break
        cnt += len(hits)
    return out[:cnt], ovf, covf


def test_per_cell_rule_equals_sequential_loop():
    rng = random.Random(20240607)
    for _ in range(30000):
        cap = rng.randint(1, 9)
        bucket_cap = rng.randint(1, 6)
        cells = []
        for lane in range(27):
            if rng.random() < 0.3:
                cells.append(None)  # empty cell (stamp mismatch)
                continue
            size = rng.randint(1, 9)
            entries = [(rng.random() < 0.4, 100 * lane + k) for k in range(min(size, bucket_cap))]
            cells.append((entries, size > bucket_cap))
        large = [(rng.random() < 0.5, 9000 + k) for k in range(rng.choice([0, 1, 2, 31, 33, 70]))]
        assert per_cell(cells, large, cap, bucket_cap) == sequential(cells, large, cap, bucket_cap)
