"""Comparison of NJ set-up results (rapidNJ::initialize outputs) for the NJ tests.

Sorted rows: std::sort leaves the order of equal distances unspecified, so
against the reference's own rows equal-distance runs are compared as sets of
(id, distance bits); a run cut by rapidNJMem's cap is compared by value only
(which ids it keeps depends on that order).  Against the oracle, which orders
ties by id like the library, rows are compared exactly.
"""
import numpy as np

ARRAYS = ("sums", "separations", "max_row_separations", "index_to_id", "redundant_to_master",
          "redundant_count", "row_lengths")


def bits(a):
    return np.asarray(a, dtype=np.float32).view(np.uint32)


def golden(z, cap):
    """The reference's results stored by tests/golden/make_golden_nj.py."""
    p = f"c{cap}_"
    r = {k: z[p + k] for k in ARRAYS}
    r["max_separation"] = np.float32(z[p + "max_separation"])
    lens, cat = z[p + "list_len"], z[p + "list_cat"]
    offs = np.concatenate([[0], np.cumsum(lens)])
    r["lists"] = [list(cat[offs[i]:offs[i + 1]]) for i in range(len(lens))]
    rows, pos = [], 0
    ids, dist = z[p + "row_ids"], z[p + "row_dist"]
    for i in range(len(lens)):
        if r["index_to_id"][i] == -1:
            rows.append(None)
            continue
        k = int(r["row_lengths"][i])
        rows.append((ids[pos:pos + k], dist[pos:pos + k]))
        pos += k
    r["rows"] = rows
    return r


def lists_from_master(master):
    """redundantMap lists from redundant_to_master: each master's other class rows,
    descending (the order of the reference's push_front in ascending j)."""
    n = len(master)
    out = [[] for _ in range(n)]
    for j in range(n - 1, -1, -1):
        if master[j] != j:
            out[master[j]].append(j)
    return out


def compare(got, want, cap, exact_ties):
    for k in ("sums", "separations", "max_row_separations"):
        assert np.array_equal(bits(got[k]), bits(want[k])), k
    for k in ("index_to_id", "redundant_to_master", "redundant_count", "row_lengths"):
        assert np.array_equal(np.asarray(got[k]), np.asarray(want[k])), k
    assert bits(got["max_separation"]) == bits(want["max_separation"])
    assert lists_from_master(got["redundant_to_master"]) == [list(x) for x in want["lists"]]
    for i, (g, w) in enumerate(zip(got["rows"], want["rows"])):
        assert (g is None) == (w is None), i
        if g is None:
            continue
        gi, gd = np.asarray(g[0], np.uint32), np.asarray(g[1], np.float32)
        wi, wd = np.asarray(w[0], np.uint32), np.asarray(w[1], np.float32)
        assert len(gi) == len(wi), i
        if exact_ties:
            assert np.array_equal(gi, wi) and np.array_equal(bits(gd), bits(wd)), i
            continue
        assert np.array_equal(gd, wd), i  # by value: -0 == +0
        k = len(gi)
        s = 0
        while s < k:
            e = s + 1
            while e < k and wd[e] == wd[s]:
                e += 1
            cut = cap > 0 and k == cap and e == k
            if not cut:
                a = sorted(zip(gi[s:e].tolist(), bits(gd[s:e]).tolist()))
                b = sorted(zip(wi[s:e].tolist(), bits(wd[s:e]).tolist()))
                assert a == b, (i, s, e)
            s = e


def device_rows(res):
    """Sorted rows of a GPU result as the oracle's list of (ids, distances)."""
    ids = res["sorted"][..., 0].cpu().numpy().view(np.uint32)
    dist = res["sorted_distances"].cpu().numpy()
    rows = []
    for i in range(len(res["index_to_id"])):
        if res["index_to_id"][i] == -1:
            rows.append(None)
        else:
            k = int(res["row_lengths"][i])
            rows.append((ids[i, :k], dist[i, :k]))
    return rows
