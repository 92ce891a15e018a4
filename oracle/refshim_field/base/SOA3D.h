// Shim (oracle test infrastructure): VecGeom's SOA3D, unused by the scalar
// field-map reader but included by it.
#pragma once
