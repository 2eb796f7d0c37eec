"""Result tables of the correlators.

The reference returns astropy.table.Table objects with columns
(k, ps, histogram, count) and (r, xi, histogram, count)
(fftcorr/correlate/correlator.pyx:42-70).  astropy is used when it is
installed; otherwise this small column table with the same names, column
order and indexing is returned.
"""
import numpy as np


class Table:
    def __init__(self, data, names):
        if len(data) != len(names):
            raise ValueError("one name per column is required")
        self._cols = {n: np.array(d, copy=True) for n, d in zip(names, data)}
        self._names = list(names)

    @property
    def colnames(self):
        return list(self._names)

    def __getitem__(self, key):
        if isinstance(key, str):
            return self._cols[key]
        return {n: c[key] for n, c in self._cols.items()}

    def __len__(self):
        return len(self._cols[self._names[0]]) if self._names else 0

    def __contains__(self, name):
        return name in self._cols

    def keys(self):
        return list(self._names)

    def __repr__(self):
        return "Table(" + ", ".join(
            f"{n}{tuple(self._cols[n].shape)}" for n in self._names) + ")"


def make_table(data, names):
    try:
        import astropy.table
    except ImportError:
        return Table(data, names)
    return astropy.table.Table(data=data, names=names, copy=True)
