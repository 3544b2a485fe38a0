"""Test oracle (not product code): the reference daemon's row rules restated in plain Python.

Engine results are pairs of distinct-geometry ids; the daemon turns them into rows of input ids
(daemon/gpujoind.cu of landstats-us/postgis-cuda):
  - a deduplicated layer's geometry g stands for its member rows midx[moff[g]:moff[g+1]] (Layer::members, :71-74);
  - op_join (:268-283) / op_dwithin (:470-481): members x members; a self-join ("same" layer, each unordered pair
    reported once) writes (ra, rb) and, off the diagonal, (rb, ra) for self_pairs "all"; for "distinct" only
    lo < hi rows, skipping a row paired with itself;
  - op_relate (:354-367): the same rules, a mirrored row carries the transposed DE-9IM code, except pairs of one
    distinct geometry with itself (identical geometries), whose rows keep the code;
  - stats-only counts (:257-267, :454-463);
  - op_cluster (:302-313): cluster numbers dense in order of first row.
"""


def members(moff, midx, g):
    if moff is None:
        return [g]
    return [int(x) for x in midx[moff[g]:moff[g + 1]]]


def pair_rows(a, b, ma, mb, same, distinct):
    """[(ra, rb, transposed)] of one engine pair; ma / mb = (moff, midx) or (None, None)."""
    out = []
    diag = same and a == b
    for ra in members(*ma, a):
        for rb in members(*mb, b):
            if not same:
                out.append((ra, rb, False))
            elif distinct:
                if ra == rb or (diag and ra > rb):
                    continue
                out.append((ra, rb, False) if ra < rb else (rb, ra, not diag))
            else:
                out.append((ra, rb, False))
                if not diag:
                    out.append((rb, ra, True))
    return out


def row_count(a, b, ma, mb, same, distinct):
    na = 1 if ma[0] is None else int(ma[0][a + 1] - ma[0][a])
    nb = 1 if mb[0] is None else int(mb[0][b + 1] - mb[0][b])
    if not same:
        return na * nb
    if a == b:
        return na * (na - 1) // 2 if distinct else na * na
    return na * nb if distinct else 2 * na * nb


def expand(pairs, ma, mb, same, distinct):
    """[(ra, rb, pair index, transposed)] for all pairs, in pair order."""
    out = []
    for i, (a, b) in enumerate(pairs):
        out.extend((ra, rb, i, t) for ra, rb, t in pair_rows(int(a), int(b), ma, mb, same, distinct))
    return out


def cluster_labels(root, moff, midx, rows):
    row_root = [0] * rows
    for g in range(len(root)):
        for r in members(moff, midx, g):
            row_root[r] = int(root[g])
    dense, out = {}, []
    for r in range(rows):
        out.append(dense.setdefault(row_root[r], len(dense)))
    return out
