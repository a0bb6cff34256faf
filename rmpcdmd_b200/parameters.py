"""Parameter files of the RMPCDMD programs (the ParseText format they read
with PTparse / PTread_*, e.g. programs/single_dimer_pbc.f90:109-193).

The format, as the reference's parameter files use it: one ``key = value``
per line; ``#`` starts a comment; a value is a single token (integer, real,
logical ``T`` / ``F``, string) or a space-separated vector.  ParseText itself
is a submodule absent from the reference tree; this reader follows the files
and the calls: ``PTread_i``, ``PTread_d``, ``PTread_l``, ``PTread_s``,
``PTread_ivec``, ``PTread_dvec``.  A missing key is an error (the calls in the
programs give no defaults), as is a vector of the wrong length.
"""
from __future__ import annotations

from pathlib import Path


class ParameterError(ValueError):
    pass


_TRUE = {"t", ".true.", "true"}
_FALSE = {"f", ".false.", "false"}


class Parameters:
    """The key / value pairs of one parameter file; ``read`` records every key
    a program read (the reference stores them in its H5MD parameters group)."""

    def __init__(self, text: str, source: str = "<string>"):
        self.source = source
        self.values: dict[str, list[str]] = {}
        self.read: dict[str, object] = {}
        for n, raw in enumerate(text.splitlines(), 1):
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            if "=" not in line:
                raise ParameterError(f"{source}:{n}: expected 'key = value', got {raw!r}")
            key, val = (x.strip() for x in line.split("=", 1))
            if not key or not val:
                raise ParameterError(f"{source}:{n}: empty key or value in {raw!r}")
            self.values[key] = val.split()

    @classmethod
    def from_file(cls, path) -> "Parameters":
        p = Path(path)
        return cls(p.read_text(), str(p))

    def _tokens(self, key: str) -> list[str]:
        if key not in self.values:
            raise ParameterError(f"{self.source}: parameter {key!r} not found")
        return self.values[key]

    def _one(self, key: str) -> str:
        t = self._tokens(key)
        if len(t) != 1:
            raise ParameterError(f"{self.source}: parameter {key!r} must be a single value, got {t}")
        return t[0]

    def _keep(self, key, v):
        self.read[key] = v
        return v

    def i(self, key: str) -> int:
        """PTread_i"""
        return self._keep(key, int(self._one(key)))

    def d(self, key: str) -> float:
        """PTread_d (Fortran exponents 1.0d-3 accepted)"""
        return self._keep(key, _real(self._one(key)))

    def l(self, key: str) -> bool:
        """PTread_l"""
        v = self._one(key).lower()
        if v in _TRUE:
            return self._keep(key, True)
        if v in _FALSE:
            return self._keep(key, False)
        raise ParameterError(f"{self.source}: parameter {key!r} is not a logical: {v!r}")

    def s(self, key: str) -> str:
        """PTread_s"""
        return self._keep(key, " ".join(self._tokens(key)))

    def ivec(self, key: str, n: int) -> list[int]:
        """PTread_ivec"""
        t = self._tokens(key)
        if len(t) != n:
            raise ParameterError(f"{self.source}: parameter {key!r} needs {n} values, got {len(t)}")
        return self._keep(key, [int(x) for x in t])

    def dvec(self, key: str, n: int) -> list[float]:
        """PTread_dvec"""
        t = self._tokens(key)
        if len(t) != n:
            raise ParameterError(f"{self.source}: parameter {key!r} needs {n} values, got {len(t)}")
        return self._keep(key, [_real(x) for x in t])


def _real(tok: str) -> float:
    return float(tok.lower().replace("d", "e"))


def format_parameters(values: dict) -> str:
    """A parameter file holding ``values`` (lists become vectors, booleans T / F)."""
    out = []
    for k, v in values.items():
        if isinstance(v, bool):
            s = "T" if v else "F"
        elif isinstance(v, (list, tuple)):
            s = " ".join(str(x) for x in v)
        else:
            s = str(v)
        out.append(f"{k} = {s}")
    return "\n".join(out) + "\n"
