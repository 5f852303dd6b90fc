"""Shim: the subset of yaff's System/Cell used on the reference's grid-solve path."""
import numpy as np

__all__ = ["Cell", "System", "Parameters", "ForceField", "log"]


class Cell(object):
    def __init__(self, rvecs):
        self.rvecs = np.asarray(rvecs, dtype=float).reshape(-1, 3)
        self.nvec = len(self.rvecs)

    @property
    def volume(self):
        return float(abs(np.linalg.det(self.rvecs)))

    @property
    def parameters(self):
        lengths = np.linalg.norm(self.rvecs, axis=1)
        angles = np.zeros(3)
        for i in range(3):
            a, b = self.rvecs[(i + 1) % 3], self.rvecs[(i + 2) % 3]
            angles[i] = np.arccos(np.clip(np.dot(a, b) / (np.linalg.norm(a) * np.linalg.norm(b)), -1, 1))
        return lengths, angles


class System(object):
    def __init__(self, numbers=None, pos=None, ffatypes=None, ffatype_ids=None, rvecs=None, masses=None):
        self.pos = None if pos is None else np.array(pos, dtype=float)
        self.ffatypes = None if ffatypes is None else list(ffatypes)
        self.ffatype_ids = None if ffatype_ids is None else np.asarray(ffatype_ids, dtype=int)
        self.cell = None if rvecs is None else Cell(rvecs)
        self.masses = masses
        self.numbers = numbers

    @property
    def natom(self):
        return 0 if self.pos is None else len(self.pos)

    @classmethod
    def from_file(cls, *args, **kwargs):
        raise NotImplementedError("shim: build hosts by setting attributes")


class Parameters(object):
    @classmethod
    def from_file(cls, *args, **kwargs):
        raise NotImplementedError("shim: pass LJ parameters as a dict")


class ForceField(object):
    pass


class _Log(object):
    silent = 0
    def set_level(self, level):
        pass


log = _Log()
