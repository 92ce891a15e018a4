#pragma once
// Shim: particle base type for IsApplicable traits.
namespace geantx { struct Particle {}; }
