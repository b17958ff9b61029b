"""The reference's on-disk array format: native binary with a SEP-style text
header (binWrite / binRead, src/include/IO.hpp:179-429; chosen by
param.format, IO.hpp:432-443).

The header lists, for each axis i = 1..ndim (axis 1 fastest), ``n<i>=``,
``o<i>=`` and ``d<i>=`` on lines of their own, then ``esize=`` (bytes per
sample) and ``in=`` (the path of the binary file, written as
``<datapath>/<header path>@``).  The binary holds the samples in native byte
order, axis 1 fastest.  Reading accepts ``label<i>=``, ``#`` comment lines
and a quoted ``in=``; trailing axes of length 1 are dropped, as binRead does
(down to ndim0 axes).

Arrays here are C-ordered numpy arrays whose LAST index is axis 1, so the
reference's model [npar][nx][nz] (z = axis 1) is an array of shape
(npar, nx, nz).
"""
import os
from typing import List, Optional, Sequence, Tuple

import numpy as np

Axis = Tuple[int, float, float, str]   # (n, o, d, label)


def _fmt(v) -> str:
    """A number as C++'s default ostream prints it (6 significant digits)."""
    if float(v) == int(v) and abs(v) < 1e6:
        return str(int(v))
    return "%g" % float(v)


def default_datapath() -> str:
    """Where binWrite puts the binary: $DATAPATH, else $PWD, else "."."""
    return os.environ.get("DATAPATH") or os.environ.get("PWD") or "."


def write_bin(array, header: str, axes: Optional[Sequence[Tuple[float, float]]] = None,
              datapath: Optional[str] = None, dtype=np.float32) -> str:
    """Write array (axis 1 = last numpy index) as binWrite does.  axes:
    optional (o, d) per reference axis, axis 1 first (default (0, 1)).
    Returns the path of the binary file."""
    a = np.ascontiguousarray(array, dtype=dtype)
    shape = list(a.shape[::-1]) or [1]
    axes = list(axes) if axes is not None else []
    lines = []
    for i, n in enumerate(shape):
        o, d = axes[i] if i < len(axes) else (0.0, 1.0)
        lines += ["n%d=%d" % (i + 1, n), "o%d=%s" % (i + 1, _fmt(o)), "d%d=%s" % (i + 1, _fmt(d))]
    binpath = (datapath if datapath is not None else default_datapath()) + "/" + header + "@"
    lines += ["esize=%d" % a.dtype.itemsize, "in=" + binpath]
    with open(header, "w") as f:
        f.write("\n".join(lines) + "\n")
    a.tofile(binpath)
    return binpath


def read_header(header: str) -> Tuple[List[Axis], int, str]:
    """Parse a header: (axes n1..n6 with o, d, label; esize; binary path)."""
    n = [1] * 6
    o = [0.0] * 6
    d = [1.0] * 6
    lab = [""] * 6
    esize, path = 4, ""
    with open(header) as f:
        for line in f:
            if line.startswith("#"):
                continue
            for w in line.split():
                key, eq, val = w.partition("=")
                if not eq:
                    continue
                if len(key) == 2 and key[0] in "nod" and key[1] in "123456":
                    k = int(key[1]) - 1
                    if key[0] == "n":
                        n[k] = int(val)
                    elif key[0] == "o":
                        o[k] = float(val)
                    else:
                        d[k] = float(val)
                elif key[:5] == "label" and key[5:] in ("1", "2", "3", "4", "5", "6"):
                    lab[int(key[5:]) - 1] = val
                elif key == "esize":
                    esize = int(val)
                elif key == "in":
                    path = val[1:-1] if val.startswith('"') else val
    return [(n[i], o[i], d[i], lab[i]) for i in range(6)], esize, path


def read_bin(header: str, ndim0: int = 1, dtype=np.float32) -> Tuple[np.ndarray, List[Axis]]:
    """Read a header and its binary as binRead does: returns (array with axis 1
    last, the kept axes).  The binary must hold exactly n1*...*n6*esize bytes;
    esize 4 or 8 is converted to dtype.  A relative in= path is taken from the
    working directory, as binRead's fopen does, else from the header's
    directory."""
    axes, esize, path = read_header(header)
    ndim = 6
    while ndim > 1 and axes[ndim - 1][0] == 1 and ndim0 != ndim:
        ndim -= 1
    axes = axes[:ndim]
    n123 = int(np.prod([a[0] for a in axes]))
    if not os.path.isabs(path) and not os.path.exists(path):
        alt = os.path.join(os.path.dirname(os.path.abspath(header)), path)
        if os.path.exists(alt):
            path = alt
    size = os.path.getsize(path)
    if size != n123 * esize:
        raise ValueError("the binary file contains %d bytes whereas the description file suggests %d bytes"
                         % (size, n123 * esize))
    if esize not in (4, 8):
        raise ValueError("esize %d: only 4 (float) and 8 (double) samples are read" % esize)
    raw = np.fromfile(path, dtype=np.float32 if esize == 4 else np.float64, count=n123)
    return raw.astype(dtype, copy=False).reshape([a[0] for a in axes][::-1]), axes
