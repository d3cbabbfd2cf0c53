"""Minimal stand-in for h5py, backed by the DQSF sim-file container.

Only what the reference generator (util/gen_1band_unified_hub.py:929-1195)
calls is provided: File(path, mode) as a context manager, create_group,
item get/set on files and groups, Dataset[...] read/write and ExternalLink.
It exists so that the generator can be run here to produce golden inputs;
nothing in the engine imports it.
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "..", "..",
                                "dqmc-dev_b200"))
from dqmc_b200 import simfile  # noqa: E402


class ExternalLink:
    def __init__(self, filename, path):
        self.filename = filename
        self.path = path


class Dataset:
    def __init__(self, f, name):
        self._f, self._name = f, name

    def __getitem__(self, key):
        v = self._f._get(self._name)
        return v if key is Ellipsis else np.asarray(v)[key]

    def __setitem__(self, key, value):
        cur = np.asarray(self._f._get(self._name))
        new = cur.copy()
        new[key] = value
        self._f._set(self._name, new.astype(cur.dtype))

    @property
    def dtype(self):
        return np.asarray(self._f._get(self._name)).dtype

    @property
    def shape(self):
        return np.asarray(self._f._get(self._name)).shape

    def __array__(self, dtype=None, copy=None):
        a = np.asarray(self._f._get(self._name))
        return a if dtype is None else a.astype(dtype)


class Group:
    def __init__(self, f, name):
        self._f, self._name = f, name

    def _path(self, key):
        return f"{self._name}/{key}" if self._name else key

    def create_group(self, key):
        self._f._groups.add(self._path(key))
        return Group(self._f, self._path(key))

    def __getitem__(self, key):
        return self._f._lookup(self._path(key))

    def __setitem__(self, key, value):
        self._f._assign(self._path(key), value)

    def __contains__(self, key):
        return self._f._exists(self._path(key))


class File(Group):
    def __init__(self, path, mode="r"):
        super().__init__(self, "")
        self._path_on_disk = path
        self._mode = mode
        self._groups = set()
        self._data = {}
        exists = os.path.exists(path)
        if mode == "x" and exists:
            raise FileExistsError(path)
        if mode in ("r", "r+", "a") and exists:
            self._data = simfile.read(path, resolve_links=False)
        elif mode in ("r", "r+"):
            raise FileNotFoundError(path)
        self._dirty = mode != "r"

    # container plumbing
    def _get(self, name):
        if name in self._data:
            return self._data[name]
        head = name.split("/")[0]
        link = self._data.get(head)
        if isinstance(link, simfile.Link):
            base = os.path.dirname(os.path.abspath(self._path_on_disk))
            return simfile.read(os.path.join(base, link.filename))[name]
        raise KeyError(name)

    def _set(self, name, value):
        self._data[name] = value

    def _exists(self, name):
        try:
            self._get(name)
            return True
        except KeyError:
            return name in self._groups or any(
                k.startswith(name + "/") for k in self._data)

    def _lookup(self, name):
        if name in self._data and not isinstance(self._data[name], simfile.Link):
            return Dataset(self, name)
        if (name in self._groups or isinstance(self._data.get(name), simfile.Link)
                or any(k.startswith(name + "/") for k in self._data)):
            return Group(self, name)
        self._get(name)
        return Dataset(self, name)

    def _assign(self, name, value):
        if isinstance(value, ExternalLink):
            self._data[name] = simfile.Link(value.filename)
        elif isinstance(value, Dataset):
            self._data[name] = np.array(value._f._get(value._name))
        else:
            self._data[name] = value

    def close(self):
        if self._dirty:
            simfile.write(self._path_on_disk, self._data)
            self._dirty = False

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False
