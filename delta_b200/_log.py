"""Logging (mirror of python/delta/_log.py): loguru, silent by default."""

from __future__ import annotations

import sys
import time
from collections.abc import Iterator
from contextlib import contextmanager

from loguru import logger

logger.disable("delta_b200")


def configure_logging(level: str = "INFO", sink=None) -> int:
    """Enable the library's log output at ``level`` (stderr by default)."""
    logger.enable("delta_b200")
    return logger.add(sink or sys.stderr, level=level, format="{time:HH:mm:ss} | {level:<7} | {message}")


@contextmanager
def log_timing(label: str) -> Iterator[None]:
    """Log '<label> done in <s>s' at INFO when the block exits."""
    t0 = time.perf_counter()
    try:
        yield
    finally:
        logger.info("{} done in {:.3f}s", label, time.perf_counter() - t0)
