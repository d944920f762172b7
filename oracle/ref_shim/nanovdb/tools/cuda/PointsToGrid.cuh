// Empty stand-in for NanoVDB's CUB-based device grid builder. The reference's kernel
// source includes it, but the host-compiled oracle never builds grids on a device, so
// this header shadows the real one on the oracle's include path.
#pragma once
