"""raymond_b200 — a B200-native wavefront path tracer behind iRath96/raymond's
scene and shader interface.  See include/raymond.h for the C ABI."""
