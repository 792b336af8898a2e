"""Environment sets in the C ABI's structure-of-arrays form (include/bcc.h).

An ``EnvSet`` holds, per primitive kind, one count per environment and the
records of all environments concatenated in environment order -- the layout
``bcc_env_soa`` points at.  Record widths follow the reference shapes
(src/collision/shapes.hh) minus their std::string header:

* sphere  4 floats: x y z r
* capsule 8 floats: x1 y1 z1 xv yv zv r rdv   (also the z-aligned capsules)
* cuboid 15 floats: x y z, axis1, axis2, axis3, h1 h2 h3 (also z-aligned)

Cylinders are carried for API fidelity only: the reference's device scan never
reads them (src/utils.cuh:213-245).
"""
import ctypes

import numpy as np

KINDS = ("spheres", "capsules", "z_capsules", "cuboids", "z_cuboids", "cylinders")
WIDTH = {"spheres": 4, "capsules": 8, "z_capsules": 8, "cuboids": 15, "z_cuboids": 15,
         "cylinders": 8}


class BccEnvSoa(ctypes.Structure):
    """Mirror of ``bcc_env_soa`` (include/bcc.h)."""
    _fields_ = [("num_envs", ctypes.c_int32)] + [
        ("num_" + k, ctypes.POINTER(ctypes.c_uint32)) for k in KINDS] + [
        (k, ctypes.POINTER(ctypes.c_float)) for k in KINDS]


def _empty(kind):
    return np.zeros((0, WIDTH[kind]), np.float32)


class EnvSet:
    def __init__(self, counts, records):
        n = None
        self.counts, self.records = {}, {}
        for k in KINDS:
            c = np.ascontiguousarray(counts.get(k, []), dtype=np.uint32)
            if n is None:
                n = len(c) if len(c) else None
            self.counts[k] = c
            r = records.get(k)
            self.records[k] = _empty(k) if r is None else np.ascontiguousarray(r, np.float32).reshape(-1, WIDTH[k])
        n = max(len(c) for c in self.counts.values())
        for k in KINDS:
            if len(self.counts[k]) == 0:
                self.counts[k] = np.zeros(n, np.uint32)
            if len(self.counts[k]) != n:
                raise ValueError("count arrays disagree on the number of environments")
            if int(self.counts[k].sum()) != len(self.records[k]):
                raise ValueError("%s: counts sum to %d but %d records given" % (
                    k, int(self.counts[k].sum()), len(self.records[k])))
        self.num_envs = n
        self._keep = None

    @staticmethod
    def from_lists(envs):
        """envs: list of dicts kind -> array [m, width] (missing kinds = none)."""
        counts = {k: [] for k in KINDS}
        recs = {k: [] for k in KINDS}
        for e in envs:
            for k in KINDS:
                r = np.asarray(e.get(k, _empty(k)), np.float32).reshape(-1, WIDTH[k])
                counts[k].append(len(r))
                recs[k].append(r)
        return EnvSet(counts, {k: (np.concatenate(v) if v else _empty(k)) for k, v in recs.items()})

    def env(self, i):
        out = {}
        for k in KINDS:
            off = int(self.counts[k][:i].sum())
            out[k] = self.records[k][off:off + int(self.counts[k][i])]
        return out

    def subset(self, idx):
        return EnvSet.from_lists([self.env(int(i)) for i in idx])

    def num_primitives(self):
        return sum(self.counts[k].astype(np.int64) for k in KINDS if k != "cylinders")

    def as_ctypes(self):
        """A BccEnvSoa pointing into this set's arrays (valid while the set lives)."""
        s = BccEnvSoa()
        s.num_envs = self.num_envs
        u32 = ctypes.POINTER(ctypes.c_uint32)
        f32 = ctypes.POINTER(ctypes.c_float)
        for k in KINDS:
            setattr(s, "num_" + k, self.counts[k].ctypes.data_as(u32))
            r = self.records[k]
            setattr(s, k, r.ctypes.data_as(f32) if len(r) else None)
        self._keep = s
        return s
