"""On-disk cache of fault-stiffness matrices, built column block by column block.

The reference rebuilds K on every run (`build_model` calls `fault_stiffness`
each time, src/BP8.jl:215-218). Here a K is stored once per key

    (grid: n1, n2, n3, extents; lam; mu; l_f; SBP order; solver tolerance;
     format version)

as column-block files plus a manifest, so a build that stops part way
resumes where it stopped and a later run with the same key loads K instead
of solving again:

    K = cached_fault_stiffness(fe, "/data/kcache")            # builds or loads
    K = cached_fault_stiffness(fe, "/data/kcache", block=512)  # block = columns per file

Layout of one entry (directory named by the key's SHA-256 prefix):
    manifest.json           key fields, nf, block size, list of finished blocks
    cols_<c0>_<c1>.npy      K[:, c0:c1] (FP64, 2nf x (c1 - c0), column-major)

Blocks are written to a temporary name and renamed, and the manifest is
rewritten after each block, so an interrupted build leaves only whole blocks.
"""
import hashlib
import json
import os
import tempfile

import numpy as np

FORMAT_VERSION = 1


def cache_key(fe, rtol=None):
    """The fields that determine K (a different value of any gives another K)."""
    g = fe.grids
    return {
        "format": FORMAT_VERSION,
        "n": [g.n1, g.n2, g.n3],
        "x1_extent": g.x1_extent, "x2": list(g.x2), "x3": list(g.x3),
        "lam": fe.lam, "mu": fe.mu, "l_f": fe.l_f,
        "sbp_order": 4,
        "rtol": fe.rs.rtol if rtol is None else float(rtol),
    }


def key_digest(key):
    return hashlib.sha256(json.dumps(key, sort_keys=True).encode()).hexdigest()[:24]


def _atomic_write(path, write):
    d = os.path.dirname(path)
    fd, tmp = tempfile.mkstemp(dir=d, prefix=".tmp_")
    os.close(fd)
    try:
        write(tmp)
        os.replace(tmp, path)
    finally:
        if os.path.exists(tmp):
            os.remove(tmp)


class KCache:
    """One cache entry for one key."""

    def __init__(self, root, key, nf, block=512):
        self.key = key
        self.nf = int(nf)
        self.dir = os.path.join(root, key_digest(key))
        os.makedirs(self.dir, exist_ok=True)
        self.mpath = os.path.join(self.dir, "manifest.json")
        if os.path.exists(self.mpath):
            m = json.load(open(self.mpath))
            if m["key"] != key or m["nf"] != self.nf:
                raise ValueError(f"cache entry {self.dir} holds a different key")
            self.block = int(m["block"])
            self.done = [tuple(b) for b in m["blocks"]]
        else:
            self.block = int(block)
            self.done = []
            self._save_manifest()

    def _save_manifest(self):
        m = {"key": self.key, "nf": self.nf, "block": self.block, "blocks": sorted(self.done)}
        _atomic_write(self.mpath, lambda p: json.dump(m, open(p, "w"), indent=1))

    def blocks(self):
        n = 2 * self.nf
        return [(c0, min(c0 + self.block, n)) for c0 in range(0, n, self.block)]

    def missing(self):
        have = set(self.done)
        return [b for b in self.blocks() if b not in have]

    def _bpath(self, b):
        return os.path.join(self.dir, f"cols_{b[0]}_{b[1]}.npy")

    def put(self, b, cols_block):
        cols_block = np.asfortranarray(cols_block, dtype=np.float64)
        if cols_block.shape != (2 * self.nf, b[1] - b[0]):
            raise ValueError(f"block {b} has shape {cols_block.shape}")
        _atomic_write(self._bpath(b), lambda p: np.save(open(p, "wb"), cols_block))
        if tuple(b) not in self.done:
            self.done.append(tuple(b))
        self._save_manifest()

    def complete(self):
        return not self.missing()

    def load(self):
        if not self.complete():
            raise ValueError(f"cache entry {self.dir} is missing {len(self.missing())} block(s)")
        n = 2 * self.nf
        K = np.empty((n, n), order="F")
        for b in self.blocks():
            K[:, b[0]:b[1]] = np.load(self._bpath(b))
        return K


def cached_fault_stiffness(fe, root, block=512, build=None, verbose=False):
    """`fault_stiffness(fe)` through the on-disk cache: load K when the entry
    is complete, otherwise build the missing column blocks (and store each
    as it finishes). `build(cols) -> (2nf, len(cols))` defaults to the GPU
    column build `stiffness_columns(fe, cols)`."""
    c = KCache(root, cache_key(fe), fe.nf, block)
    todo = c.missing()
    if build is None:
        from . import stiffness_columns
        build = lambda cols: stiffness_columns(fe, cols)[0]  # noqa: E731
    for b in todo:
        cols = np.arange(b[0], b[1], dtype=np.int32)
        c.put(b, build(cols))
        if verbose:
            print(f"kcache: columns {b[0]}:{b[1]} of {2 * fe.nf} stored in {c.dir}")
    return c.load()
