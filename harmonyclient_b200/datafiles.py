"""Dataset, result-file and recall utilities of the reference's benchmark
driver, restated for numpy callers (src/utils.h:187-407 loaders, 565-620
result files, 622-756 recall metrics; src/utils.h:41-140 and
src/stats.h:122-134 the CSV rows).  They read and write the same files the
reference does and return the same numbers, so a user of the reference's
`query` / `main` tools finds the same inputs and metrics here.

Files, as the reference reads them:

* ``.fvecs``: records ``[int32 d][d float32]``; n = file size // (4 + 4d).
* ``.bvecs``: the reference's loader takes the file's first int32 as d, then
  reads record i's d bytes from offset ``8 + i (4 + d)`` and counts
  ``(size - 4) // (4 + d)`` records (src/utils.h:286-320): the layout of a
  4-byte file header followed by ``[int32 d][d uint8]`` records.
  ``bvecs_records=True`` reads the plain record layout instead (the first
  record at offset 4).  The info function counts ``size // (4 + d)`` records
  (src/utils.h:268-282), as the reference does.
* ``.txt``: one vector per line, comma separated, the first field skipped;
  d = the number of values on the first line; the loader ignores row bounds
  when reached through load_xvecs (src/utils.h:373-386).
* result files: ``.txt`` (one line per query, ``label distance`` pairs, six
  decimals) or binary (nq*k int64 labels, then nq*k float32 distances).
"""
import os

import numpy as np

METRIC_IP, METRIC_L2 = 0, 1
FEPS = 1e-4


# ---------------------------------------------------------------------------
# vector files
def _first_int(path):
    with open(path, "rb") as f:
        return int(np.frombuffer(f.read(4), np.int32)[0])


def load_xvecs_info(path):
    """(n, d) as loadXvecsInfo counts them (src/utils.h:186-283, 328-338)."""
    path = str(path)
    if path.endswith(".fvecs"):
        d = _first_int(path)
        return os.path.getsize(path) // (4 + d * 4), d
    if path.endswith(".bvecs"):
        d = _first_int(path)
        return os.path.getsize(path) // (4 + d), d
    if path.endswith(".txt"):
        m, d = 0, 0
        with open(path) as f:
            for line in f:
                line = line.rstrip("\n")
                if m == 0:
                    d = len(line.split(",")) - 1
                m += 1
        return m, d
    raise ValueError("no support file")


def _bounds(a, b, bmax):
    b = bmax if b == 0 else b
    if not (a >= 1 and b <= bmax and b >= a):
        raise ValueError(f"row bounds {a}..{b} outside 1..{bmax}")
    return a, b


def load_fvecs(path, bounds=(1, 0)):
    """Rows a..b (1-based, inclusive; b = 0: to the end) of an .fvecs file
    (src/utils.h:203-235)."""
    d = _first_int(path)
    rec = 4 + 4 * d
    bmax = os.path.getsize(path) // rec
    a, b = _bounds(bounds[0], bounds[1], bmax)
    raw = np.fromfile(path, np.uint8, count=(b - a + 1) * rec, offset=(a - 1) * rec)
    return raw.reshape(b - a + 1, rec)[:, 4:].copy().view(np.float32)


def load_bvecs(path, bounds=(1, 0), bvecs_records=False):
    """Rows a..b of a .bvecs file as uint8 (src/utils.h:285-320).  Reads the
    reference's layout (record i's bytes at 8 + i(4+d)) unless
    bvecs_records=True (at 4 + i(4+d))."""
    d = _first_int(path)
    rec = 4 + d
    size = os.path.getsize(path)
    if bvecs_records:
        bmax, start = size // rec, 4
    else:
        bmax, start = (size - 4) // rec, 8
    a, b = _bounds(bounds[0], bounds[1], bmax)
    n = b - a + 1
    # Only the bytes of rows a..b are read: record i's d bytes sit at
    # start + i*rec, so rows a..b span n records from start + (a-1)*rec (the
    # last record's trailing 4 bytes may lie past the end of the file).
    off = start + (a - 1) * rec
    want = n * rec
    raw = np.fromfile(path, np.uint8, count=min(want, size - off), offset=off)
    if raw.size < want:
        raw = np.concatenate([raw, np.zeros(want - raw.size, np.uint8)])
    return raw.reshape(n, rec)[:, :d].copy()


def bvecs_is_records(path):
    """True when a .bvecs file holds plain ``[int32 d][d uint8]`` records
    (size a multiple of 4 + d, the layout of the public BIGANN files), False
    when it has the reference loader's extra 4-byte header (size - 4 a
    multiple of 4 + d).  Raises ValueError when it is neither."""
    d = _first_int(path)
    size = os.path.getsize(path)
    if d <= 0:
        raise ValueError(f"{path}: first int32 {d} is not a dimension")
    if size % (4 + d) == 0:
        return True
    if (size - 4) % (4 + d) == 0:
        return False
    raise ValueError(f"{path}: size {size} fits neither [int32 d][d bytes] records nor the reference's "
                     f"4-byte header before them (d = {d})")


def bvecs_rows(path, bvecs_records):
    """Rows in a .bvecs file of the given layout."""
    d = _first_int(path)
    size = os.path.getsize(path)
    return size // (4 + d) if bvecs_records else (size - 4) // (4 + d)


def load_tvecs(path, bounds=(1, 0)):
    """Rows of a comma-separated .txt file, the first field of each line
    skipped (src/utils.h:339-386)."""
    rows = []
    with open(path) as f:
        for line in f:
            vals = line.rstrip("\n").split(",")[1:]
            rows.append([float(v) for v in vals])
    m = len(rows)
    d = len(rows[0]) if rows else 0
    a, b = _bounds(bounds[0], bounds[1], m)
    return np.array([r[:d] for r in rows[a - 1:b]], np.float32).reshape(b - a + 1, d)


def load_xvecs(path, bounds=(1, 0), bvecs_records=False):
    """float32 rows of .fvecs, .bvecs (converted) or .txt (every row: the
    reference's loadXvecs passes no bounds to the text loader)
    (src/utils.h:388-399).  bvecs_records as in load_bvecs."""
    path = str(path)
    if path.endswith(".fvecs"):
        return load_fvecs(path, bounds)
    if path.endswith(".bvecs"):
        return load_bvecs(path, bounds, bvecs_records).astype(np.float32)
    if path.endswith(".txt"):
        return load_tvecs(path)
    raise ValueError("no support file")


def write_fvecs(path, x):
    """[int32 d][d float32] records."""
    x = np.ascontiguousarray(x, np.float32)
    n, d = x.shape
    rec = np.empty((n, 1 + d), np.float32)
    rec[:, 0] = np.array([d], np.int32).view(np.float32)[0]
    rec[:, 1:] = x
    rec.tofile(path)


def write_bvecs(path, x, bvecs_records=False):
    """[int32 d][d uint8] records; with the reference's layout (default) the
    file starts with one more int32 d, so load_bvecs reads it back whole."""
    x = np.ascontiguousarray(x, np.uint8)
    n, d = x.shape
    rec = np.empty((n, 4 + d), np.uint8)
    rec[:, :4] = np.frombuffer(np.array([d], np.int32).tobytes(), np.uint8)
    rec[:, 4:] = x
    with open(path, "wb") as f:
        if not bvecs_records:
            f.write(np.array([d], np.int32).tobytes())
        f.write(rec.tobytes())


# ---------------------------------------------------------------------------
# result files (src/utils.h:565-620)
def write_results(labels, distances, path):
    labels = np.ascontiguousarray(labels, np.int64)
    distances = np.ascontiguousarray(distances, np.float32)
    nq, k = labels.shape
    path = str(path)
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    if path.endswith("txt"):
        with open(path, "w") as f:
            for i in range(nq):
                f.write(" ".join(f"{int(labels[i, j])} {float(distances[i, j]):.6f}" for j in range(k)) + "\n")
    else:
        with open(path, "wb") as f:
            f.write(labels.tobytes())
            f.write(distances.tobytes())


def load_results(path, nq, k):
    path = str(path)
    if path.endswith("txt"):
        tok = open(path).read().split()
        labels = np.array([int(t) for t in tok[0:2 * nq * k:2]], np.int64).reshape(nq, k)
        dist = np.array([float(t) for t in tok[1:2 * nq * k:2]], np.float32).reshape(nq, k)
        return labels, dist
    raw = np.fromfile(path, np.uint8, count=nq * k * 12)
    labels = raw[:nq * k * 8].view(np.int64).reshape(nq, k).copy()
    dist = raw[nq * k * 8:].view(np.float32).reshape(nq, k).copy()
    return labels, dist


# ---------------------------------------------------------------------------
# recall metrics (src/utils.h:622-756)
def relative_error(x, y):
    x, y = np.float32(x), np.float32(y)
    return abs(y) if x == 0 else abs((x - y) / x)


def _gt_sets(GT, nq, k, gt_k):
    return [set(int(v) for v in GT.reshape(-1)[i * gt_k:i * gt_k + k]) for i in range(nq)]


def calculate_recall(I, D, GT, GD, nq, k, metric, gt_k=0):
    """Fraction of returned ids found among the first k ground-truth ids of
    their query (src/utils.h:661-732; its consistency assert is compiled out
    in Release builds)."""
    I, D = np.asarray(I, np.int64).reshape(-1), np.asarray(D, np.float32).reshape(-1)
    if D[0] < 0:
        return 0.0
    gt_k = gt_k or k
    if k > gt_k:
        raise ValueError("k should be less than or equal to gt_k.")
    sets = _gt_sets(np.asarray(GT, np.int64), nq, k, gt_k)
    hit = 0
    for i in range(nq):
        for j in range(k):
            v = int(I[i * k + j])
            if v == -1:
                break
            hit += v in sets[i]
    return float(np.float32(hit) / np.float32(nq * k))


def calculate_recall_loose(I, D, GT, GD, nq, k, metric, gt_k=0):
    """Like calculate_recall, a returned entry also counting when its
    distance is below the k-th ground-truth distance or within 1e-4 of it
    (src/utils.h:631-658; that distance is read at GD[i*k + k-1])."""
    I, D = np.asarray(I, np.int64).reshape(-1), np.asarray(D, np.float32).reshape(-1)
    GD = np.asarray(GD, np.float32).reshape(-1)
    gt_k = gt_k or k
    if D[0] < 0:
        return 0.0
    if k > gt_k:
        raise ValueError("k should be less than or equal to gt_k.")
    sets = _gt_sets(np.asarray(GT, np.int64), nq, k, gt_k)
    hit = 0
    for i in range(nq):
        max_dis = GD[i * k + k - 1]
        for j in range(k):
            v = int(I[i * k + j])
            if v == -1:
                break
            dv = D[i * k + j]
            if v in sets[i] or dv < max_dis or abs(dv - max_dis) <= FEPS:
                hit += 1
    return float(np.float32(hit) / np.float32(nq * k))


def calculate_r2(I, D, GT, GD, nq, k, metric, gt_k=0):
    """Sum of returned distances over the sum of the ground truth's, minus 1,
    over the entries up to each query's first -1 (src/utils.h:734-756; f32
    sums in query-major order)."""
    I, D = np.asarray(I, np.int64).reshape(-1), np.asarray(D, np.float32).reshape(-1)
    GD = np.asarray(GD, np.float32).reshape(-1)
    gt_k = gt_k or k
    if k > gt_k:
        raise ValueError("k should be less than or equal to gt_k.")
    g_sum, s = np.float32(0), np.float32(0)
    for i in range(nq):
        for j in range(k):
            if I[i * k + j] == -1:
                break
            g_sum = np.float32(g_sum + GD[i * gt_k + j])
            s = np.float32(s + D[i * k + j])
    return float(np.float32(s / g_sum) - np.float32(1))


# ---------------------------------------------------------------------------
# CSV rows (src/utils.h:41-140, src/stats.h:122-134)
STATS_COLUMNS = ["dataset", "mode", "nb", "nq", "d", "nlist", "nprobe", "k", "divideIVF", "orderOptimize",
                 "UnblockSend", "cut", "block", "worker", "group", "team", "time_speedup", "query_time",
                 "original_time", "recall", "r2", "variance", "train_time", "add_time", "preSearch_time", "ratio",
                 "teamRatio", "brute_ratio"]


def csv_field(v):
    """One value as the reference's CsvWriter prints it: float32 with 7
    decimals, float64 with 16 (std::fixed, digits10 + 1), bool as 1 / 0."""
    if isinstance(v, (bool, np.bool_)):
        return "1" if v else "0"
    if isinstance(v, np.float32):
        return f"{float(v):.7f}"
    if isinstance(v, (float, np.float64)):
        return f"{float(v):.16f}"
    return str(v)


def append_csv_row(path, values, columns=STATS_COLUMNS, append=True):
    """Writes the header first unless appending to an existing file."""
    new = not (append and os.path.exists(path))
    with open(path, "a" if not new else "w") as f:
        if new:
            f.write(",".join(columns) + "\n")
        f.write(",".join(csv_field(v) for v in values) + "\n")
