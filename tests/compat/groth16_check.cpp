// A program in the shape of the reference's test/groth16.cu, built against
// liblzk_b200 through include/lzk_compat.hpp: the same three calls, then one
// machine-readable line with the proof's 256-byte wire form for the test.
#include <cstdio>
#include <cstdlib>
#include "lzk_compat.hpp"

using namespace lzk_compat;

int main(int argc, char** argv)
{
    uint64_t seed = argc > 1 ? std::strtoull(argv[1], nullptr, 10) : 1;
    Groth16_BN254 protocol(input_scale::MatMul_p_39, seed);
    protocol.Setup(12);
    protocol.Prove();
    std::printf("WIRE");
    for (uint32_t w : protocol.wire()) std::printf(" %08x", w);
    std::printf("\n");
    return protocol.wire().empty() ? 1 : 0;
}
