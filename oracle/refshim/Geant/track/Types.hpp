// Shim (oracle test infrastructure): the reference's track/Types.hpp pulls in
// VecGeom's navigation state through core/Typedefs.hpp; the event and vertex
// containers (source/Geant/proxy/ProxyVertex.hpp) need only ThreeVector and
// TrackState from it, which the shim TrackState provides.
#pragma once
#include "Geant/track/TrackState.hpp"
#ifndef REQUIRE
#define REQUIRE(x) ((void)0)
#endif
