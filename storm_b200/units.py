"""CGS constants (CODATA 2018) the problem builders hand to the engine through
the descriptor.  The oracle's `units` stand-in holds the same values; a test
checks they agree bit for bit."""

_clight = 2.99792458e10          # cm/s
_k_boltz = 1.380649e-16          # erg/K
_kev = 1.602176634e-9            # erg
_sigma_sb = 5.670374419e-5       # erg/(cm^2 s K^4)

UNITS = {
    "clight": _clight,
    "k_boltz": _k_boltz,
    "kev": _kev,
    "kev_kelvin": _kev / _k_boltz,
    "sigma_sb": _sigma_sb,
    "arad": 4.0 * _sigma_sb / _clight,
}
