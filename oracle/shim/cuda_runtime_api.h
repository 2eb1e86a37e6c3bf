/* Host-only stand-in (see shim/cuda.h); nothing from the runtime is needed. */
#pragma once
