"""FITS provenance cards describing the software environment."""

from __future__ import annotations

import platform


def environment_cards() -> dict[str, object]:
    from . import __version__

    cards: dict[str, object] = {"DLTVER": __version__, "DLTPY": platform.python_version(), "DLTENGN": "b200-sm100a"}
    try:
        import numpy

        cards["DLTNPY"] = numpy.__version__
    except ImportError:  # pragma: no cover
        pass
    return cards
