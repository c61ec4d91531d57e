// lbvh_mid.hpp -- placed after the reference's __device__ globals (split_count,
// level_split_count) and before its host recursion: the reference reads the
// split count with a string-named cudaMemcpyFromSymbol, replaced here by a
// direct read of the same global. TEST INFRASTRUCTURE ONLY.
static inline uint host_get_split_count() { return split_count; }
