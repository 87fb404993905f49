"""Errors of the kriging engine, named as the reference's (python/boitata/errors.py)."""


class InvalidInput(ValueError):
    """Invalid parameters or data (the reference's boitata.errors.InvalidInput)."""


class Unsupported(InvalidInput):
    """A reference option this engine does not run on the GPU."""
