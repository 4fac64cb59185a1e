// C entry points onto the reference's CPU Hilbert functions
// (src/serialize/hilbert.cu, CPU::hilbert_encode / CPU::hilbert_decode), so
// that the oracle's restatement can be checked against them.  Test
// infrastructure only; compiled by oracle/build.py together with the
// reference source file into oracle/_ref.
#include <cstddef>
#include <cstdint>

#include "hilbert.h"

extern "C" void ref_hilbert_encode(size_t n, const uint32_t *x, const uint32_t *y, const uint32_t *z, uint32_t *codes)
{
    CPU::hilbert_encode(n, x, y, z, codes);
}

extern "C" void ref_hilbert_decode(size_t n, const uint32_t *codes, uint32_t *x, uint32_t *y, uint32_t *z)
{
    CPU::hilbert_decode(n, codes, x, y, z);
}
