"""B200-native SDF-to-mesh engine (see include/sdfmesh_b200.h for the C ABI)."""
