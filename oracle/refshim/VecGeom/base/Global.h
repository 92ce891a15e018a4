// Shim (oracle test infrastructure): the few standard headers and the host
// attribute the reference's hot-path sources expect from VecGeom.
#pragma once
#include <cassert>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#define VECCORE_ATT_HOST_DEVICE
