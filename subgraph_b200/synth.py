"""Synthetic benchmark inputs in the reference's own file formats, made with
numpy alone (this module never loads the native library, so the reference's
CPU program can be run on the same files without it).

  rmat_edges     seeded R-MAT graph: edge_factor * 2^scale draws with the
                 initiator (a, b, c, 1-a-b-c), vertex ids scrambled by a random
                 permutation, self loops dropped, each undirected edge kept
                 once as (min, max), sorted; the largest id in use is renamed
                 2^scale - 1 so that the reference's edge-list reader keeps all
                 2^scale vertices (it renumbers only when the largest id is not
                 V - 1, EdgeList.cpp:70-113).
  write_edge_list  the reference's text format "V\\nE\\nu v\\n..." (read by
                 EdgeList::readfromEdgeList, EdgeList.cpp:34-116).
  rmat_file      both, cached on disk by (scale, edge factor, initiator, seed).

The draws come from numpy's PCG64 stream, not from graph500's generator; the
sizes, initiator and degree distribution are those of the reference's
benchmark graphs (graph500 make_graph, make_graph.h:21-35), not its exact
edges.
"""
from __future__ import annotations

import hashlib
import os
import tempfile

import numpy as np


def rmat_edges(scale: int, edge_factor: int, seed: int = 1, a: float = 0.57, b: float = 0.19,
               c: float = 0.19) -> tuple[int, np.ndarray, np.ndarray]:
    """(V, src, dst) of a seeded undirected R-MAT graph, src < dst, sorted."""
    if not 1 <= scale <= 30:
        raise ValueError("scale must be in [1, 30]")
    V = 1 << scale
    E = edge_factor * V
    rng = np.random.Generator(np.random.PCG64(seed))
    # quadrant thresholds on uniform 32-bit draws
    t_a, t_ab, t_abc = (np.uint32(min(int(x * 2.0**32), 2**32 - 1)) for x in (a, a + b, a + b + c))
    us, vs = [], []
    step = 1 << 22
    for lo in range(0, E, step):
        n = min(step, E - lo)
        u = np.zeros(n, np.uint32)
        v = np.zeros(n, np.uint32)
        for _ in range(scale):
            r = rng.integers(0, 1 << 32, size=n, dtype=np.uint32)
            u <<= 1
            u |= r >= t_ab                           # quadrants c and d: lower half for the source
            v <<= 1
            v |= ((r >= t_a) & (r < t_ab)) | (r >= t_abc)   # quadrants b and d: right half for the target
        us.append(u)
        vs.append(v)
    perm = rng.permutation(V).astype(np.int64)
    u = perm[np.concatenate(us)]
    v = perm[np.concatenate(vs)]
    keep = u != v
    u, v = u[keep], v[keep]
    key = np.minimum(u, v) * V + np.maximum(u, v)

    def dedupe(k):
        k.sort()
        if len(k) > 1:
            k = k[np.concatenate(([True], k[1:] != k[:-1]))]
        return k

    key = dedupe(key)
    lo_, hi_ = key // V, key % V
    top = int(hi_.max()) if len(hi_) else V - 1
    if top != V - 1:                             # V - 1 is unused: give its id to the largest one in use
        lo_ = np.where(lo_ == top, V - 1, lo_)
        hi_ = np.where(hi_ == top, V - 1, hi_)
        key = dedupe(np.minimum(lo_, hi_) * V + np.maximum(lo_, hi_))
        lo_, hi_ = key // V, key % V
    return V, lo_.astype(np.int32), hi_.astype(np.int32)


def write_edge_list(path: str, V: int, src: np.ndarray, dst: np.ndarray) -> None:
    """Writes "V\\nE\\n" then one "u v" line per edge (atomically: temp file + rename)."""
    import pyarrow as pa
    import pyarrow.csv as pacsv
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=d, suffix=".part")
    try:
        with os.fdopen(fd, "wb") as f:
            f.write(f"{V}\n{len(src)}\n".encode())
            table = pa.table({"u": pa.array(src, pa.int32()), "v": pa.array(dst, pa.int32())})
            pacsv.write_csv(table, f, write_options=pacsv.WriteOptions(include_header=False, delimiter=" ",
                                                                        quoting_style="none"))
        os.replace(tmp, path)
    except BaseException:
        if os.path.exists(tmp):
            os.unlink(tmp)
        raise


def cache_dir() -> str:
    return os.environ.get("SUBGRAPH_B200_INPUTS", os.path.join(tempfile.gettempdir(), "subgraph_b200_inputs"))


def rmat_file(scale: int, edge_factor: int, seed: int = 1, a: float = 0.57, b: float = 0.19,
              c: float = 0.19) -> str:
    """Path of the text edge list of rmat_edges(...), generated on first use."""
    name = f"rmat_s{scale}_ef{edge_factor}_a{a:g}_b{b:g}_c{c:g}_seed{seed}.txt"
    path = os.path.join(cache_dir(), name)
    if not os.path.exists(path):
        V, src, dst = rmat_edges(scale, edge_factor, seed, a, b, c)
        write_edge_list(path, V, src, dst)
    return path


def edges_digest(V: int, src: np.ndarray, dst: np.ndarray) -> str:
    """SHA-256 over V and the int32 edge arrays: identifies a generated graph."""
    h = hashlib.sha256()
    h.update(np.int64(V).tobytes())
    h.update(np.ascontiguousarray(src, np.int32).tobytes())
    h.update(np.ascontiguousarray(dst, np.int32).tobytes())
    return h.hexdigest()
