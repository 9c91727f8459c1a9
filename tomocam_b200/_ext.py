"""Import of the compiled ``cTomocam`` module with a clear error when unbuilt."""
try:
    from . import cTomocam  # noqa: F401
except ImportError as e:  # pragma: no cover
    raise ImportError("tomocam_b200.cTomocam is not built: run `python -m tomocam_b200.build` "
                      f"({e})") from e
