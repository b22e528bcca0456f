/*
 * Stand-in for OpenMM's SFMT generator interface (oracle harness only).  OpenMM's SFMT
 * (a SIMD Mersenne twister) is not available here.  This generator keeps the same interface
 * (init_gen_rand, genrand_real2 returning a double in [0, 1), checkpoint save/load) but its
 * stream is splitmix64: state += 0x9E3779B97F4A7C15, mixed by the published splitmix64
 * finaliser (Steele, Lea, Flood 2014), and genrand_real2 = (z >> 11) * 2^-53.  The oracle's C
 * restatement reproduces this stream exactly in its "sequential" random mode, so the two
 * CPU implementations can be compared bit for bit also with fluctuations and noise.
 */
#ifndef SHIM_SFMT_H_
#define SHIM_SFMT_H_
#include <cstdint>
#include <istream>
#include <ostream>
namespace OpenMM_SFMT {
class SFMT {
public:
    SFMT() : state(0) {}
    uint64_t state;
    void createCheckpoint(std::ostream& stream) { stream.write((const char*) &state, sizeof(state)); }
    void loadCheckpoint(std::istream& stream) { stream.read((char*) &state, sizeof(state)); }
};
inline void init_gen_rand(uint32_t seed, SFMT& sfmt) { sfmt.state = (uint64_t) seed; }
inline double genrand_real2(SFMT& sfmt) {
    sfmt.state += 0x9E3779B97F4A7C15ULL;
    uint64_t z = sfmt.state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z = z ^ (z >> 31);
    return (double) (z >> 11) * (1.0/9007199254740992.0);
}
}
#endif
