/* Linux stand-in for <Windows.h> as used by the reference's minimum_lbvh.h
 * (minimum_lbvh.h:18): only InterlockedExchange is needed, by build_lbvh
 * (minimum_lbvh.h:335). A sequentially consistent exchange, as on Windows.
 * Test infrastructure only (oracle/_ref). */
#pragma once
#include <stdint.h>
template <class T, class U>
static inline T InterlockedExchange(T* target, U value)
{
    return __atomic_exchange_n(target, (T)value, __ATOMIC_SEQ_CST);
}
