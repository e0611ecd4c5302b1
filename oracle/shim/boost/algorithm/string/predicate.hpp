/* Shim: included by BioBloomMaker/BloomFilterGenerator.cpp, which uses none
 * of its functions. */
#ifndef BBT_SHIM_BOOST_PREDICATE_HPP
#define BBT_SHIM_BOOST_PREDICATE_HPP
#endif
