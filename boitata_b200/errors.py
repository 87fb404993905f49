"""Errors of the kriging engine, named as the reference's (python/boitata/errors.py)."""


class BoitataError(Exception):
    """Base of every error the engine raises (the reference's boitata.errors.BoitataError)."""


class InvalidInput(BoitataError, ValueError):
    """Invalid parameters or data (the reference's boitata.errors.InvalidInput)."""


class MissingColumn(BoitataError, KeyError):
    """A column name the container or table does not hold; the message lists those it holds."""

    __str__ = Exception.__str__


class Unsupported(InvalidInput):
    """A reference option this engine does not run on the GPU."""
