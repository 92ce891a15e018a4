// Shim (oracle test infrastructure): VecGeom's base/Global.h for the
// reference's CMS field-map reader (examples/magneticfield/simplifiedCMS).
#pragma once
#include <cmath>
#include <cstdio>
