"""Make the reference's Python package importable on this interpreter, in a scratch copy.

The reference (LupoLab/solprop) targets Python 3.14; this image has 3.12. Four
mechanical edits make its NumPy backend (`numpy_ref`) import and run here, and
nothing else about its arithmetic changes:

1. ``except A, B:`` (PEP 758 syntax) becomes ``except (A, B):``.
2. ``from __future__ import annotations`` is inserted after each module docstring,
   because 3.14 defers annotation evaluation and the sources rely on it.
3. ``typing.get_protocol_members`` (3.13) is aliased to typing_extensions'.
4. ``h5py`` and ``optmat`` are stubbed: neither is installed, and neither is on
   the propagation path once species data are supplied by the caller.

The copy is written under a temporary directory, never into this repository.
This script is test infrastructure: it only serves the fixture generator beside it.
"""

from __future__ import annotations

import ast
import os
import re
import shutil
import sys
import tempfile
import types
from pathlib import Path

REFERENCE = Path(os.environ.get("SOLPROP_REFERENCE", "/root/reference"))
_EXCEPT = re.compile(r"^(\s*)except ([A-Za-z_][\w.]*(?:\s*,\s*[A-Za-z_][\w.]*)+)(\s+as\s+\w+)?\s*:")


def _rewrite(text: str) -> str:
    lines = text.splitlines(keepends=True)
    out = []
    for line in lines:
        m = _EXCEPT.match(line)
        if m and " as " not in m.group(2):
            indent, names, alias = m.group(1), m.group(2), m.group(3) or ""
            line = f"{indent}except ({names}){alias}:" + line[m.end():]
        out.append(line)
    text = "".join(out)
    if "from __future__ import annotations" in text:
        return text
    try:
        tree = ast.parse(text)
    except SyntaxError:
        return text
    insert_at = 0
    if tree.body and isinstance(tree.body[0], ast.Expr) and isinstance(
        getattr(tree.body[0], "value", None), ast.Constant
    ) and isinstance(tree.body[0].value.value, str):
        insert_at = tree.body[0].end_lineno
    src_lines = text.splitlines(keepends=True)
    src_lines.insert(insert_at, "from __future__ import annotations\n")
    return "".join(src_lines)


def build(target: Path | None = None) -> Path:
    """Write the backported copy and return the directory to put on ``sys.path``."""
    target = Path(target or Path(tempfile.gettempdir()) / "solprop_backport")
    stamp = target / ".stamp"
    if stamp.exists():
        return target
    if target.exists():
        shutil.rmtree(target)
    src = REFERENCE / "src" / "solprop"
    for path in src.rglob("*"):
        rel = path.relative_to(src.parent)
        dest = target / rel
        if path.is_dir():
            dest.mkdir(parents=True, exist_ok=True)
            continue
        dest.parent.mkdir(parents=True, exist_ok=True)
        if path.suffix == ".py":
            dest.write_text(_rewrite(path.read_text()))
        else:
            shutil.copy2(path, dest)
    stamp.write_text("ok")
    return target


def install_shims() -> None:
    """Alias the 3.13 typing API and stub the two absent packages."""
    import typing

    import typing_extensions

    if not hasattr(typing, "get_protocol_members"):
        typing.get_protocol_members = typing_extensions.get_protocol_members
    if "h5py" not in sys.modules:
        sys.modules["h5py"] = types.ModuleType("h5py")
    if "optmat" not in sys.modules:
        optmat = types.ModuleType("optmat")
        optmat.__version__ = "0+stub"
        sys.modules["optmat"] = optmat


def activate() -> None:
    """Build the copy if needed, install the shims and make ``solprop`` importable."""
    install_shims()
    path = build()
    if str(path) not in sys.path:
        sys.path.insert(0, str(path))


if __name__ == "__main__":
    activate()
    import solprop  # noqa: F401

    print("solprop importable from", build())
