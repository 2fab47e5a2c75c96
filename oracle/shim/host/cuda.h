// Empty stand-in for <cuda.h> when the reference projector sources are compiled
// for the host CPU (see host_shim.h).
#pragma once
