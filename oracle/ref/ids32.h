// ORACLE -- TEST INFRASTRUCTURE ONLY.
// Forced include for building the reference from its own sources on Linux.
// The reference was written for MSVC, where uint_fast32_t is 4 bytes; its cell
// arithmetic relies on that width (iindx + indxx.y * cN.x wraps modulo 2^32,
// md_interaction_list_reconstructbpm.cu:99-118). With glibc's 8-byte
// uint_fast32_t the negative octant offsets land outside pnC. This header gives
// the reference build the 4-byte id type its author's toolchain uses.
#pragma once
#include <stdint.h>
#ifdef __cplusplus
#include <cstdint>
#endif
#define uint_fast32_t uint32_t
#undef UINT_FAST32_MAX
#define UINT_FAST32_MAX UINT32_MAX
