/*
 * shim_binomial.cpp -- TEST INFRASTRUCTURE ONLY.  Exposes the Boost binomial
 * stand-in (shim/boost/math/distributions/binomial.hpp), through the same
 * calls the reference makes (Common/SeqEval.h:199-216,
 * BioBloomCategorizer/MIBFClassifier.hpp:930-939), to the CPU tests that check
 * it against scipy.stats.binom.
 */
#include <boost/math/distributions/binomial.hpp>

using namespace boost::math::policies;
using namespace boost::math;
typedef binomial_distribution<double, policy<discrete_quantile<integer_round_up> > > binom_round_up;

extern "C" double shim_binom_sf(unsigned n, double p, unsigned x)
{
	binom_round_up bin(n, p);
	return cdf(complement(bin, x));
}

extern "C" unsigned shim_binom_quantile(unsigned n, double p, double q)
{
	binom_round_up bin(n, p);
	unsigned i = quantile(complement(bin, q));
	return i;
}
