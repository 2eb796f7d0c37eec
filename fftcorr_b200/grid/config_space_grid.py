"""ConfigSpaceGrid with its data resident in GPU memory.

Mirrors fftcorr/grid/config_space_grid.pyx:10-207 (constructor validation,
cell-size choice, properties, in-place arithmetic, clear, to_grid_coords,
ASDF write/read) over the C++ grid of cc/grid/config_space_grid.h:10-57.

The authoritative copy of the grid lives on the device, where MassAssignor
writes it and the correlators read it without any host transfer.  ``.data``
returns a float64 numpy array that mirrors it: the first access turns the
mirror on, after which the mirror is refreshed after every device-side change
and uploaded before every device-side use, so in-place numpy edits such as
``dens -= mean`` behave like edits of the reference's aliased view.

Extension beyond the reference: a keyword-only ``precision`` ("fp64", the
default and the reference's type, or "fp32").  An FP32 grid stores FP32
cells, which the FP32-mixed correlators read directly; mass assignment still
sums in FP64 and rounds once per update of a cell, and ``.data`` is still a
float64 mirror.
"""
import ctypes

import numpy as np

from fftcorr_b200 import _lib

_CELL_PRECISIONS = {"fp64": _lib.FC_FP64, "fp32": _lib.FC_FP32_MIXED}


def _cell_precision(precision):
    if precision not in _CELL_PRECISIONS:
        raise ValueError(f"precision must be 'fp64' or 'fp32', got {precision!r}")
    return _CELL_PRECISIONS[precision]


class ConfigSpaceGrid:
    def __init__(self, shape, posmin, posmax, cell_size=None, padding=0,
                 extra_pad=0, metadata=None, *, precision="fp64"):
        prec = _cell_precision(precision)
        shape = np.ascontiguousarray(shape, dtype=np.intc)
        posmin = np.asarray(posmin, dtype=np.double).copy(order="C")
        posmax = np.asarray(posmax, dtype=np.double).copy(order="C")
        if shape.shape != (3,):
            raise ValueError(
                "Expected shape to have shape (3,), got: {}".format(shape.shape))
        if np.any(shape <= 0):
            raise ValueError("Expected shape to be positive, got: {}".format(shape))
        if posmin.shape != (3,):
            raise ValueError(
                "Expected posmin to have shape (3,), got: {}".format(posmin.shape))
        if posmax.shape != (3,):
            raise ValueError(
                "Expected posmax to have shape (3,), got: {}".format(posmax.shape))
        if np.any(posmax <= posmin):
            raise ValueError(
                "Expected posmin < posmax, got posmin={}, posmax={}".format(
                    posmin, posmax))
        if cell_size is not None and cell_size <= 0:
            raise ValueError(
                "Expected cell_size to be positive, got: {}".format(cell_size))
        if padding < 0:
            raise ValueError("Expected padding > 0, got {}".format(padding))
        if extra_pad < 0:
            raise ValueError("Expected extra_pad > 0, got {}".format(extra_pad))
        if extra_pad:
            print("Padding boundaries by {:.6g}".format(extra_pad))
            posmin -= extra_pad
            posmax += extra_pad
        minimum_cell_size = np.amax((posmax - posmin) / shape)
        if cell_size is not None:
            print("Requested cell size {:.6g}".format(cell_size))
            if cell_size < minimum_cell_size:
                raise ValueError(
                    "Requested cell size too small to cover entire region. "
                    "Need at least {:.6g}".format(minimum_cell_size))
        else:
            cell_size = minimum_cell_size
        posmax = posmin + shape * cell_size
        print("Adopting:")
        print("  shape = [" + ", ".join(["{}".format(x) for x in shape]) + "]")
        print("  cell_size = {:.6g}".format(cell_size))
        print("  posmin = [" + ", ".join(["{:.6g}".format(x) for x in posmin]) + "]")
        print("  posmax = [" + ", ".join(["{:.6g}".format(x) for x in posmax]) + "]")
        for arr in (posmin, posmax):
            arr.setflags(write=False)
        self._shape = tuple(int(s) for s in shape)
        self._posmin = posmin
        self._posmax = posmax
        self._cell_size = float(cell_size)
        self._padding = padding + extra_pad
        self._metadata = {}
        if metadata:
            self._metadata.update(metadata)
        self._handle = None
        self._host = None
        self._mirror = False
        self._precision = precision
        h = ctypes.c_void_p()
        _lib.call("fc_grid_create_precision", _lib.iptr(shape), _lib.dptr(posmin),
                  self._cell_size, prec, ctypes.byref(h))
        self._handle = h

    @classmethod
    def from_geometry(cls, shape, posmin, cell_size, metadata=None, *,
                      precision="fp64"):
        """A grid with posmin and cell size given directly (no printing)."""
        prec = _cell_precision(precision)
        self = cls.__new__(cls)
        shape = np.ascontiguousarray(shape, dtype=np.intc)
        posmin = np.asarray(posmin, dtype=np.double).copy(order="C")
        self._shape = tuple(int(s) for s in shape)
        self._posmin = posmin
        self._posmax = posmin + shape * cell_size
        self._posmin.setflags(write=False)
        self._posmax.setflags(write=False)
        self._cell_size = float(cell_size)
        self._padding = 0
        self._metadata = dict(metadata or {})
        self._host = None
        self._mirror = False
        self._precision = precision
        h = ctypes.c_void_p()
        _lib.call("fc_grid_create_precision", _lib.iptr(shape), _lib.dptr(posmin),
                  self._cell_size, prec, ctypes.byref(h))
        self._handle = h
        return self

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.load().fc_grid_destroy(h)
            except Exception:
                pass
            self._handle = None

    # -------------------------------------------------- device coherence
    @property
    def handle(self):
        return self._handle

    def _before_device(self):
        """Uploads host-side edits before device work reads the grid."""
        if self._mirror:
            _lib.call("fc_grid_upload", self._handle, _lib.dptr(self._host))

    def _after_device(self):
        """Refreshes the host mirror after device work changed the grid."""
        if self._mirror:
            _lib.call("fc_grid_download", self._handle, _lib.dptr(self._host))

    def device_ptr(self):
        """Device address of the cells (FP64, or FP32 for an FP32 grid)."""
        p = ctypes.c_void_p()
        _lib.call("fc_grid_device_data", self._handle, ctypes.byref(p))
        return p.value

    @property
    def precision(self):
        return self._precision

    # ------------------------------------------------------- properties
    @property
    def shape(self):
        return self._shape

    @property
    def posmin(self):
        return self._posmin

    @property
    def posmax(self):
        return self._posmax

    @property
    def cell_size(self):
        return self._cell_size

    @property
    def padding(self):
        return self._padding

    @property
    def metadata(self):
        return self._metadata

    @property
    def data(self):
        if not self._mirror:
            self._host = np.empty(self._shape, dtype=np.float64)
            _lib.call("fc_grid_download", self._handle, _lib.dptr(self._host))
            self._mirror = True
        return self._host

    def __array__(self, dtype=None, copy=None):
        d = self.data
        return d if dtype is None else d.astype(dtype)

    # --------------------------------------------------------- methods
    def clear(self):
        _lib.call("fc_grid_clear", self._handle)
        if self._mirror:
            self._host[...] = 0.0
        self._metadata.clear()

    def to_grid_coords(self, survey_coords, periodic_wrap=False):
        survey_coords = np.asarray(survey_coords, dtype=np.float64)
        sc = np.ascontiguousarray(survey_coords.reshape(3))
        out = np.empty(3)
        inside = ctypes.c_int()
        _lib.call("fc_grid_coords", self._handle, _lib.dptr(sc),
                  int(bool(periodic_wrap)), _lib.dptr(out), ctypes.byref(inside))
        if not inside.value:
            raise ValueError(f"Coordinates {survey_coords} out of bounds")
        return out.reshape(survey_coords.shape)

    def sum_sumsq(self):
        """(sum, sum of squares) of the grid in FP64 (array_ops.cc:95-137)."""
        self._before_device()
        s, q = ctypes.c_double(), ctypes.c_double()
        _lib.call("fc_grid_sum", self._handle, ctypes.byref(s), ctypes.byref(q))
        return s.value, q.value

    def add_grid(self, other, scale=1.0):
        """self += scale * other, on the device."""
        self._before_device()
        other._before_device()
        _lib.call("fc_grid_axpy", self._handle, float(scale), other._handle)
        self._after_device()
        return self

    def _scalar_op(self, name, value):
        self._before_device()
        _lib.call(name, self._handle, float(value))
        self._after_device()

    def write(self, filename, dtype=np.float32):
        import asdf  # optional dependency, as in the reference
        tree = {
            "header": {
                "shape": self.shape,
                "posmin": self.posmin,
                "posmax": self.posmax,
                "cell_size": self.cell_size,
                "padding": self.padding,
            },
            "data": self.data.astype(dtype),
            "metadata": self.metadata,
        }
        with asdf.AsdfFile(tree) as af:
            af.write_to(filename)

    @classmethod
    def read(cls, filename):
        import asdf
        with asdf.open(filename) as af:
            header = af.tree["header"]
            grid = cls(shape=header["shape"], posmin=header["posmin"],
                       posmax=header["posmax"], padding=header["padding"],
                       metadata=af.tree.get("metadata"))
            assert np.allclose(grid.cell_size, header["cell_size"])
            np.copyto(grid.data, af.tree["data"])
        return grid

    def __iadd__(self, other):
        if np.isscalar(other) and not self._mirror:
            self._scalar_op("fc_grid_add_scalar", other)
        else:
            np.add(self.data, other, out=self.data)
        return self

    def __isub__(self, other):
        if np.isscalar(other) and not self._mirror:
            self._scalar_op("fc_grid_add_scalar", -other)
        else:
            np.subtract(self.data, other, out=self.data)
        return self

    def __imul__(self, other):
        if np.isscalar(other) and not self._mirror:
            self._scalar_op("fc_grid_multiply_by", other)
        else:
            np.multiply(self.data, other, out=self.data)
        return self

    def __itruediv__(self, other):
        np.divide(self.data, other, out=self.data)
        return self
