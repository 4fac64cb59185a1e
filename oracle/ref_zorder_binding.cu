// C entry points onto the reference's CPU z-order functions
// (src/serialize/z_order.cu, CPU::z_order_encode / CPU::z_order_decode), so
// that the oracle's restatement can be checked against them.  Test
// infrastructure only; compiled by oracle/build.py together with the
// reference source file into oracle/_ref.
#include <cstddef>
#include <cstdint>

#include "z_order.h"

extern "C" void ref_z_order_encode(size_t n, const uint32_t *x, const uint32_t *y, const uint32_t *z, uint32_t *codes)
{
    CPU::z_order_encode(n, x, y, z, codes);
}

extern "C" void ref_z_order_decode(size_t n, const uint32_t *codes, uint32_t *x, uint32_t *y, uint32_t *z)
{
    CPU::z_order_decode(n, codes, x, y, z);
}
