/* Shim: sdsl-lite is not installed here.  The reference's MIBFGen.hpp
 * includes this header but uses none of it directly; the bit vector and rank
 * support behind MIBloomFilter are restated in mibf_oracle.c. */
#ifndef BBT_SHIM_SDSL_INT_VECTOR_HPP
#define BBT_SHIM_SDSL_INT_VECTOR_HPP
#endif
