"""ParFlow input-database (``.pfidb``) writer.

The format is the flat key/value file that ParFlow's ``IDB_NewDB``
(pfsimulator/parflow_lib/input_database.c:76) parses: the number of entries on
the first line, then for every entry the key length, the key, the value
length and the value, one per line (the same layout pftools writes in
pftools/python/parflow/tools/io.py:1322 ``write_dict_as_pfidb``).
"""

from __future__ import annotations

import os


def _fmt(value) -> str:
    if isinstance(value, bool):
        return "True" if value else "False"
    if isinstance(value, float):
        return repr(value)
    if isinstance(value, (list, tuple)):
        return " ".join(_fmt(v) for v in value)
    return str(value)


def write_pfidb(keys: dict, path: str) -> None:
    """Write ``keys`` (a flat ``{"Dotted.Key": value}`` dict) to ``path``."""
    items = [(k, _fmt(v)) for k, v in keys.items()]
    with open(path, "w") as out:
        out.write(f"{len(items)}\n")
        for k, v in items:
            out.write(f"{len(k)}\n{k}\n{len(v)}\n{v}\n")


def read_pfidb(path: str) -> dict:
    """Read a ``.pfidb`` file back into a dict of strings."""
    with open(path) as f:
        lines = f.read().split("\n")
    n = int(lines[0])
    out = {}
    pos = 1
    for _ in range(n):
        key = lines[pos + 1]
        val = lines[pos + 3]
        out[key] = val
        pos += 4
    return out


__all__ = ["write_pfidb", "read_pfidb"]
