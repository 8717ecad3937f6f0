"""MD_PREC_FX32's split of each list row into a near row and a far row, read back through md_nlist_fx32_rows and
checked against the split rule restated here on the reference-ordered rows of md_nlist_download.

The rule: near row = the entries whose pair was closer than sqrt(near2) at the build, in row order (when there are
more than 16, the 16 closest of the first 48), then the last entries of the far part in row order up to the next
multiple of 8, then sentinels; far row = every other entry in row order, then sentinels to a multiple of 8;
groups = (near groups, far groups) of 8. The kernels classify on float frames, so a row holding a pair within
1e-5 (relative) of the radius, or whose 16th and 17th closest near pairs are that close, is checked only for
what holds either way: near and far rows together hold the row's entries, each exactly once, and the far row keeps
row order. Liquid and compressed-solid states (rows with more than 16 near entries, which k_rows_split_fix
redoes), and the split made inside md_run's CUDA graphs at a device-side rebuild.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MASK = (1 << 27) - 1
NEAR_CAP, FIX_NEAR = 16, 48
TOL = 1e-5


def prepared(md, cells, density, seed=5):
    s = md.fcc_system(cells, density, 2.0, seed=seed)
    nl = md.NeighbourList(2.5, 0.3)
    nl.build(s)
    warm = md.LennardJonesForceField(1.0, 1.0, 2.5)
    warm.compute_forces(s, nl)
    md.VelocityVerletIntegrator(0.005).run(s, warm, nl, 300, record=False)
    nl.build(s)  # positions now are the build's positions
    return s, nl


def full_rows(nl, n):
    """Each particle's row in the list's order: its own pairs (j > i, candidate order), then the j < i that list it,
    in increasing j."""
    d = nl.download()
    off, nb = d["offsets"].astype(np.int64), d["neighbours"].astype(np.int64)
    rows = [list(nb[off[i]:off[i + 1]]) for i in range(n)]
    for j in range(n):
        for k in nb[off[j]:off[j + 1]]:
            rows[k].append(j)
    return rows


def squared_distances(pos, box, i, js):
    d = pos[i, :3][None, :] - pos[js, :3]
    d -= box * np.round(d / box)
    return (d * d).sum(axis=1)


def expected_split(row, r2, near2, n):
    near = [k for k in range(len(row)) if r2[k] < near2]
    if len(near) > NEAR_CAP:
        near = sorted(sorted(near[:FIX_NEAR], key=lambda k: (r2[k], k))[:NEAR_CAP])
    chosen = set(near)
    far = [k for k in range(len(row)) if k not in chosen]
    near_len = (len(near) + 7) // 8 * 8
    take = min(near_len - len(near), len(far))
    near_row = [row[k] for k in near] + [row[k] for k in far[len(far) - take:]]
    near_row += [n] * (near_len - len(near_row))
    far_row = [row[k] for k in far[:len(far) - take]]
    far_len = (len(far_row) + 7) // 8 * 8
    far_row += [n] * (far_len - len(far_row))
    return near_row, far_row, (near_len // 8, far_len // 8)


def ambiguous(r2, near2):
    """A pair within float rounding of the radius, or of the 16th closest near pair's distance, where it matters."""
    if np.any(np.abs(r2 - near2) < TOL * near2):
        return True
    cand = np.sort(r2[np.flatnonzero(r2 < near2)[:FIX_NEAR]])
    return len(cand) > NEAR_CAP and cand[NEAR_CAP] - cand[NEAR_CAP - 1] < TOL * near2


def is_subsequence(sub, seq):
    it = iter(seq)
    return all(any(x == y for y in it) for x in sub)


def check_rows(rows, split, n, cap, pos=None, box=None):
    """Returns (rows checked against the rule, rows with more than 16 near entries among them)."""
    near2 = split["near2"]
    exact = over = 0
    for i, row in enumerate(rows):
        ng, fg = (int(x) for x in split["groups"][i])
        assert 0 <= ng <= NEAR_CAP // 8 and 0 <= 8 * fg <= cap, (i, ng, fg)
        near_row = [int(e) & MASK for e in split["near"][i, :8 * ng]]
        far_row = [int(e) & MASK for e in split["far"][i, :8 * fg]]
        real = [j for j in near_row + far_row if j != n]
        assert sorted(real) == sorted(int(j) for j in row), i
        assert len(set(real)) == len(real), i
        assert is_subsequence([j for j in far_row if j != n], [int(j) for j in row]), i
        if pos is None:
            continue
        r2 = squared_distances(pos, box, i, np.asarray(row, dtype=np.int64)) if row else np.zeros(0)
        if ambiguous(r2, near2):
            continue
        want_near, want_far, want_groups = expected_split([int(j) for j in row], r2, near2, n)
        assert (near_row, far_row, (ng, fg)) == (want_near, want_far, want_groups), i
        exact += 1
        over += int(np.count_nonzero(r2 < near2) > NEAR_CAP)
    return exact, over


@pytest.mark.parametrize("cells,density", [(12, 0.8442), (10, 1.3)])
def test_fx32_split_rows_follow_the_rule(md, cells, density):
    s, nl = prepared(md, cells, density)
    ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=md.PREC_FX32)
    with pytest.raises(md.MDError):  # no split before MD_PREC_FX32 forces on this build
        nl.fx32_rows()
    ff.compute_forces(s, nl)
    split = nl.fx32_rows()
    assert split["near2"] == pytest.approx((1.2 + 0.3) ** 2)
    n = s.n
    st = s.download()
    exact, over = check_rows(full_rows(nl, n), split, n, nl.layout()["row_capacity"], st["pos"], s.box)
    print("fx32 split", cells, density, "rows", n, "checked exactly", exact, "with >16 near", over)
    assert exact >= 0.95 * n
    if density > 1.0:
        assert over >= 0.5 * n  # the compressed solid's rows take the closest 16


def test_fx32_split_rows_after_graph_rebuilds(md):
    """The split md_run's graphs make at each device-side rebuild: after 150 steps with rebuilds, the near and far rows
    of the last build hold its rows' entries once each, with the far rows in row order; and they equal the rows of
    the host loop's split after the same steps."""
    base = md.fcc_system(12, 0.8442, 1.3, seed=5)
    st, box = base.download(), base.box
    runs = []
    for chunk in (64, 0):
        s = md.System.from_arrays(st["pos"], box, vel=st["vel"])
        s.set_graph(chunk)
        nl = md.NeighbourList(2.5, 0.3)
        ff = md.LennardJonesForceField(1.0, 1.0, 2.5, precision=md.PREC_FX32)
        nl.build(s)
        ff.compute_forces(s, nl)
        md.VelocityVerletIntegrator(0.005).run(s, ff, nl, 150)
        assert nl.rebuild_count > 5
        runs.append((s, nl, nl.fx32_rows()))
    (s, nl, split), (_, _, host) = runs
    assert s.graph_info()["launches"] == 3
    check_rows(full_rows(nl, s.n), split, s.n, nl.layout()["row_capacity"])
    assert np.array_equal(split["groups"], host["groups"])
    # the slots the groups cover (slots past them keep whatever an earlier build left)
    slots = np.arange(split["far"].shape[1])[None, :]
    assert np.array_equal(np.where(slots[:, :NEAR_CAP] < 8 * split["groups"][:, :1], split["near"], 0),
                          np.where(slots[:, :NEAR_CAP] < 8 * host["groups"][:, :1], host["near"], 0))
    assert np.array_equal(np.where(slots < 8 * split["groups"][:, 1:], split["far"], 0),
                          np.where(slots < 8 * host["groups"][:, 1:], host["far"], 0))


def test_fx32_split_rows_ragged(md):
    """A ragged start: 1,001 particles (the last 32-row group of the interleaved layouts part full) at uneven
    density, one of them alone in a hole (an empty row: no near and no far groups)."""
    base = md.fcc_system(8, 0.8442, 1.0, seed=3)
    box, pos = base.box, base.download()["pos"][:, :3]
    centre = np.full(3, box / 2)
    d = pos - centre
    d -= box * np.round(d / box)
    rng = np.random.default_rng(9)
    keep = rng.choice(np.flatnonzero((d * d).sum(axis=1) > 4.0 ** 2), 1000, replace=False)
    p = np.zeros((1001, 4))
    p[:1000, :3] = pos[keep]
    p[1000, :3] = centre
    s = md.System.from_arrays(p, box)
    nl = md.NeighbourList(2.5, 0.3)
    nl.build(s)
    md.LennardJonesForceField(1.0, 1.0, 2.5, precision=md.PREC_FX32).compute_forces(s, nl)
    split = nl.fx32_rows()
    n = s.n
    rows = full_rows(nl, n)
    exact, _ = check_rows(rows, split, n, nl.layout()["row_capacity"], s.download()["pos"], s.box)
    assert exact >= 0.95 * n
    empty = [i for i, r in enumerate(rows) if not r]
    assert empty and all(tuple(split["groups"][i]) == (0, 0) for i in empty)
