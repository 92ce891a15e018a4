#pragma once
// Shim: logging is not used on the hot path.
