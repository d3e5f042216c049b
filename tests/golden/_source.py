"""Where the fixture generators find the MOSE source tree: the first
command-line argument, else the MOSE_SOURCE_DIR environment variable."""
from __future__ import annotations

import os


def source_tree(root: str | None = None) -> str:
    root = root or os.environ.get("MOSE_SOURCE_DIR")
    if not root:
        raise SystemExit("give the MOSE source tree as the first argument or in MOSE_SOURCE_DIR")
    return root
