/* Linux stand-in for the MSVC <intrin.h> that the reference's minimum_lbvh.h
 * includes on its host path (minimum_lbvh.h:16). Test infrastructure only:
 * it lets oracle/_ref compile the reference's CPU code unchanged with g++. */
#pragma once
#include <x86intrin.h>
#include <stdint.h>
static inline unsigned int __lzcnt(unsigned int x) { return _lzcnt_u32(x); }
