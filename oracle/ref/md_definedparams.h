// ORACLE -- TEST INFRASTRUCTURE ONLY.
// The reference includes md_definedparams.h (md_braziltest_simple2.cu:10,
// md_uniaxialcompression3_simple.cu:10) but the file is not in its tree; the
// kernels built here use nothing from it.
#pragma once
