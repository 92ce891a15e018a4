// Shim (oracle test infrastructure): the field unit of the reference's map
// reader.  GeantV's own units are not vendored; the harness reads tesla.
#pragma once
namespace fieldUnits {
constexpr double tesla = 1.0;
}
