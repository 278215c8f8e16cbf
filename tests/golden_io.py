"""Loader of the golden fixtures under tests/golden/ (written by
oracle/ref/make_golden.cu from the reference's own code)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
_DT = {"u1": np.uint8, "u4": np.uint32, "u8": np.uint64}


class Fixtures:
    def __init__(self, sub):
        self.dir = os.path.join(GOLDEN, sub)
        self.index = {}
        for fn in os.listdir(self.dir):
            if fn.startswith("manifest_"):
                for line in open(os.path.join(self.dir, fn)):
                    name, dt, cnt = line.split()
                    self.index[name] = (_DT[dt], int(cnt))

    def __contains__(self, name):
        return name in self.index

    def __getitem__(self, name):
        dt, cnt = self.index[name]
        a = np.fromfile(os.path.join(self.dir, name + ".bin"), dtype=dt)
        assert a.size == cnt, name
        return a


def fixtures(sub):
    return Fixtures(sub)


def have(sub):
    return os.path.isdir(os.path.join(GOLDEN, sub))
