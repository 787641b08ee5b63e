"""Minimal STAR file reader/writer (host side).

Covers the STAR syntax the reference's parameter files use
(bsoft/src/util/rwstar.cpp): ``data_`` blocks holding ``_tag value`` items
and ``loop_`` tables, ``#`` comments, single/double quoted values.
"""
from __future__ import annotations

import os
import shlex
from dataclasses import dataclass, field


@dataclass
class StarLoop:
    tags: list = field(default_factory=list)
    rows: list = field(default_factory=list)

    def index(self, tag: str) -> int:
        try:
            return self.tags.index(tag)
        except ValueError:
            return -1

    def column(self, tag: str):
        i = self.index(tag)
        return None if i < 0 else [r[i] for r in self.rows]


@dataclass
class StarBlock:
    name: str
    items: dict = field(default_factory=dict)
    loops: list = field(default_factory=list)

    def has(self, tag: str) -> bool:
        return tag in self.items

    def real(self, tag: str, default: float = 0.0) -> float:
        v = self.items.get(tag)
        if v is None:
            return default
        try:
            return float(v)
        except ValueError:
            return default

    def integer(self, tag: str, default: int = 0) -> int:
        v = self.items.get(tag)
        if v is None:
            return default
        try:
            return int(float(v))
        except ValueError:
            return default

    def loop_with(self, tag: str):
        for lp in self.loops:
            if tag in lp.tags:
                return lp
        return None


def _tokens(line: str):
    try:
        return shlex.split(line, comments=False, posix=True)
    except ValueError:
        return line.split()


def read_star(path: str) -> list[StarBlock]:
    blocks: list[StarBlock] = []
    cur: StarBlock | None = None
    loop: StarLoop | None = None
    in_header = False
    with open(path, "r") as f:
        for raw in f:
            line = raw.strip()
            if not line or line.startswith("#"):
                if not line and loop is not None and not in_header and loop.rows:
                    loop = None
                continue
            if line.startswith("data_"):
                cur = StarBlock(line[5:])
                blocks.append(cur)
                loop = None
                continue
            if cur is None:
                continue
            if line.startswith("loop_"):
                loop = StarLoop()
                cur.loops.append(loop)
                in_header = True
                continue
            if line.startswith("_"):
                if loop is not None and in_header:
                    loop.tags.append(line.split()[0][1:])
                    continue
                loop = None
                toks = _tokens(line)
                tag = toks[0][1:]
                cur.items[tag] = toks[1] if len(toks) > 1 else ""
                continue
            if loop is not None:
                in_header = False
                toks = _tokens(line)
                if len(toks) == len(loop.tags):
                    loop.rows.append(toks)
                continue
    return blocks


def _fmt(v) -> str:
    if isinstance(v, float):
        return repr(float(v))
    s = str(v)
    if not s or any(c.isspace() for c in s):
        return "'" + s + "'"
    return s


def write_star(path: str, blocks: list[StarBlock]) -> None:
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write("# Written by bsoft_b200\n\n")
        for b in blocks:
            f.write(f"data_{b.name}\n\n")
            width = max([len(t) for t in b.items] + [10])
            for k, v in b.items.items():
                f.write(f"_{k:<{width}} {_fmt(v)}\n")
            f.write("\n")
            for lp in b.loops:
                f.write("loop_\n")
                for t in lp.tags:
                    f.write(f"_{t}\n")
                for r in lp.rows:
                    f.write(" ".join(_fmt(x) for x in r) + "\n")
                f.write("\n")
    os.replace(tmp, path)
