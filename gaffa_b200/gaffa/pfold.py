"""Folding of dedispersed series and spectra (python/gaffa/pfold.py)."""
from __future__ import annotations

from ._core import (DedispersedResult, DedispersedSpectrum, FoldedProfile, FoldResult, _fold_dedispersed_profile,
                    _fold_dedispersed_spectrum)


def fold_profile(dedispersed: DedispersedResult, *, period: float, nbin: int, dm_index: int = 0) -> FoldedProfile:
    """Integrated profile of row dm_index of a dedispersed result."""
    if dm_index < 0:
        raise ValueError("dm_index must be non-negative")
    return _fold_dedispersed_profile(dedispersed.data, tsamp=dedispersed.tsamp, period=period, nbin=nbin,
                                     dm_index=dm_index)


def fold_spectrum(spectrum: DedispersedSpectrum, *, period: float, nbin: int, tsubint: float = 10.0,
                  nsubband: int | None = None) -> FoldResult:
    """Subint x channel x phase cube of an aligned spectrum and its projections."""
    if nsubband is not None and nsubband <= 0:
        raise ValueError("nsubband must be positive")
    return _fold_dedispersed_spectrum(spectrum.data, tsamp=spectrum.tsamp, period=period, nbin=nbin,
                                      tsubint=tsubint, output_channels=0 if nsubband is None else nsubband)


def fold(data, *, period: float, nbin: int, dm_index: int = 0, tsubint: float = 10.0,
         nsubband: int | None = None):
    """fold_profile for a DedispersedResult, fold_spectrum for a DedispersedSpectrum."""
    if isinstance(data, DedispersedResult):
        return fold_profile(data, period=period, nbin=nbin, dm_index=dm_index)
    if isinstance(data, DedispersedSpectrum):
        return fold_spectrum(data, period=period, nbin=nbin, tsubint=tsubint, nsubband=nsubband)
    raise TypeError("fold expects a DedispersedResult or DedispersedSpectrum")


__all__ = ["fold", "fold_profile", "fold_spectrum"]
