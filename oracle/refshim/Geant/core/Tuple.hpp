#pragma once
// Shim: tuple metaprogramming is not used on the hot path.
#include <tuple>
#include <type_traits>
