// Stand-in for the `units` module STORM clones unpinned (install_deps.sh:61).
// CGS values from CODATA 2018 (exact SI definitions of c, k_B, e; sigma_SB
// derived).  The engine takes these constants through its problem descriptor,
// so host physics, this oracle and the device always agree.
#ifndef STORM_SHIM_UNITS_HPP
#define STORM_SHIM_UNITS_HPP
namespace units {
constexpr double clight = 2.99792458e10;            // cm / s
constexpr double clight2 = clight * clight;
constexpr double inv_clight2 = 1.0 / clight2;
constexpr double k_boltz = 1.380649e-16;            // erg / K
constexpr double kev = 1.602176634e-9;              // erg
constexpr double kev_kelvin = kev / k_boltz;        // K per keV
constexpr double sigma_sb = 5.670374419e-5;         // erg / (cm^2 s K^4)
constexpr double arad = 4.0 * sigma_sb / clight;    // erg / (cm^3 K^4)
} // namespace units
#endif
