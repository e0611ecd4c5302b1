/* Shim: the subset of boost::math::binomial_distribution that the reference
 * uses (Common/SeqEval.h:199-216, BioBloomCategorizer/MIBFClassifier.hpp:
 * 897-938, 1123-1133): pdf, cdf, cdf(complement(d, k)) and
 * quantile(complement(d, q)) under the integer_round_up discrete-quantile
 * policy.
 *
 * Definitions used (restated from the binomial distribution itself):
 *   pdf(d, i)                  = C(n,i) p^i (1-p)^(n-i), evaluated in log space
 *   cdf(complement(d, x))      = P(X > x) = sum_{i=x+1..n} pdf(i), summed from
 *                                the top of the tail down
 *   quantile(complement(d, q)) = the smallest integer x with P(X > x) <= q
 *                                (the continuous upper quantile rounded up),
 *                                which is scipy.stats.binom.isf(q, n, p).
 */
#ifndef BBT_SHIM_BINOMIAL_HPP
#define BBT_SHIM_BINOMIAL_HPP
#include <cmath>

namespace boost {
namespace math {
namespace policies {
enum discrete_quantile_policy_type {
	real, integer_round_outwards, integer_round_inwards, integer_round_down,
	integer_round_up, integer_round_nearest
};
template <discrete_quantile_policy_type N = integer_round_outwards>
struct discrete_quantile {};
template <class... A> struct policy {};
}

template <class RealType = double, class Policy = policies::policy<> >
class binomial_distribution {
public:
	binomial_distribution(RealType n = 1, RealType p = 0.5) : m_n(n), m_p(p) {}
	RealType trials() const { return m_n; }
	RealType success_fraction() const { return m_p; }
private:
	RealType m_n, m_p;
};
typedef binomial_distribution<double> binomial;

template <class D, class R> struct complemented2_type {
	complemented2_type(const D &d, const R &r) : dist(d), param(r) {}
	const D &dist;
	R param;
};
template <class D, class R>
inline complemented2_type<D, R> complement(const D &d, const R &r) {
	return complemented2_type<D, R>(d, r);
}

namespace bbt_shim_detail {
inline double binom_pmf(double n, double p, double i) {
	if (i < 0 || i > n)
		return 0.0;
	if (p <= 0.0)
		return i == 0 ? 1.0 : 0.0;
	if (p >= 1.0)
		return i == n ? 1.0 : 0.0;
	double lg = std::lgamma(n + 1) - std::lgamma(i + 1) - std::lgamma(n - i + 1)
			+ i * std::log(p) + (n - i) * std::log1p(-p);
	return std::exp(lg);
}
/* P(X > x) for integer x, summed from the top of the tail down. */
inline double binom_sf(double n, double p, double x) {
	double tail = 0.0;
	for (double i = n; i > x; i -= 1.0)
		tail += binom_pmf(n, p, i);
	return tail;
}
}

template <class R, class P, class T>
inline double pdf(const binomial_distribution<R, P> &d, const T &k) {
	return bbt_shim_detail::binom_pmf(d.trials(), d.success_fraction(), double(k));
}
template <class R, class P, class T>
inline double cdf(const binomial_distribution<R, P> &d, const T &k) {
	return 1.0 - bbt_shim_detail::binom_sf(d.trials(), d.success_fraction(), std::floor(double(k)));
}
template <class R, class P, class T>
inline double cdf(const complemented2_type<binomial_distribution<R, P>, T> &c) {
	return bbt_shim_detail::binom_sf(c.dist.trials(), c.dist.success_fraction(),
			std::floor(double(c.param)));
}
template <class R, class P, class T>
inline double quantile(const complemented2_type<binomial_distribution<R, P>, T> &c) {
	const double n = c.dist.trials(), p = c.dist.success_fraction();
	const double q = double(c.param);
	double x = n, tail = 0.0;
	while (x > 0) {
		double t = tail + bbt_shim_detail::binom_pmf(n, p, x);
		if (t > q)
			break;
		tail = t;
		x -= 1.0;
	}
	return x;
}
}
}
#endif
