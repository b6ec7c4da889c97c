"""SIGPROC filterbank reading (python/gaffa/io/__init__.py)."""
from ._core import Filterbank, FilterbankHeader

__all__ = ["Filterbank", "FilterbankHeader"]
