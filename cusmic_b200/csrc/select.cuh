// Order-statistic networks on float64, usable on host and device.
//
// Fast paths use compare-exchange networks whose unused outputs the
// compiler removes, so a "sort then read the middle" template becomes a pruned
// selection network.  They agree with the reference's stable odd-even
// transposition sort (src/sort.cuh:18-36) on every NaN-free window: the k-th
// order statistic of a multiset is unique up to the sign of a zero, and the
// sign of a zero median never reaches a mask or a pixel (medians only feed
// threshold tests, and every zero compares equal).  Windows holding a NaN take
// window_median_exact(), which reproduces the reference's NaN behaviour.
#pragma once
#include "common.cuh"

namespace cb {

// Compare-exchange as one predicate and two selects: on B200 this form
// measured 1.3x the throughput of fmin/fmax on float64 (NaN-free inputs, where
// both give the same values).
CB_HD void cas(double &a, double &b)
{
	bool swap = b < a;
	double lo = swap ? b : a, hi = swap ? a : b;
	a = lo;
	b = hi;
}

CB_HD double dmin(double a, double b)
{
	return b < a ? b : a;
}

CB_HD double dmax(double a, double b)
{
	return a < b ? b : a;
}

CB_HD double med3(double a, double b, double c)
{
	return dmax(dmin(a, b), dmin(dmax(a, b), c));
}

// Batcher's odd-even merge sort for any N: the comparators of the next power
// of two that touch an index >= N are dropped, which is the same as padding
// with +inf.  Template recursion keeps every index a compile-time constant.
template <int N, int P, int K> struct BatcherPass {
	CB_HD static void run(double (&v)[N])
	{
#pragma unroll
		for (int j = K % P; j + K < N; j += 2 * K) {
#pragma unroll
			for (int i = 0; i < K; ++i) {
				if (i + j + K < N && (i + j) / (2 * P) == (i + j + K) / (2 * P))
					cas(v[i + j], v[i + j + K]);
			}
		}
		BatcherPass<N, P, K / 2>::run(v);
	}
};
template <int N, int P> struct BatcherPass<N, P, 0> {
	CB_HD static void run(double (&)[N]) {}
};
template <int N, int P, bool Done = (P >= N)> struct BatcherDriver;
template <int N, int P> struct BatcherDriver<N, P, true> {
	CB_HD static void run(double (&)[N]) {}
};
template <int N, int P> struct BatcherDriver<N, P, false> {
	CB_HD static void run(double (&v)[N])
	{
		BatcherPass<N, P, P>::run(v);
		BatcherDriver<N, P * 2>::run(v);
	}
};

template <int N> CB_HD void sort_network(double (&v)[N])
{
	BatcherDriver<N, 1>::run(v);
}

// Middle element of a NaN-free window (pruned network).
template <int N> CB_HD double median_network(double (&v)[N])
{
	sort_network(v);
	return v[N / 2];
}

// Ascending sort of five values with nine compare-exchanges (an optimal
// network; checked by the 0-1 principle over all 32 binary inputs).
CB_HD void sort5(double &a, double &b, double &c, double &d, double &e)
{
	cas(a, b);
	cas(d, e);
	cas(c, e);
	cas(c, d);
	cas(b, e);
	cas(a, d);
	cas(a, c);
	cas(b, d);
	cas(b, c);
}

// Median of a NaN-free 3 x 3 window in row-major order: sort the columns,
// then the median is med3(max of minima, med3 of middles, min of maxima).
CB_HD double median9(double a0, double a1, double a2, double a3, double a4, double a5,
	double a6, double a7, double a8)
{
	cas(a0, a3); cas(a3, a6); cas(a0, a3);
	cas(a1, a4); cas(a4, a7); cas(a1, a4);
	cas(a2, a5); cas(a5, a8); cas(a2, a5);
	double lo = dmax(dmax(a0, a1), a2);
	double hi = dmin(dmin(a6, a7), a8);
	double mid = med3(a3, a4, a5);
	return med3(lo, mid, hi);
}

// The middle slot after the reference's odd-even transposition sort, for any
// window (NaNs included).  That exchange never moves a NaN and never crosses
// one, so NaNs stay put and split the window into segments that are sorted
// independently and stably; n phases sort any segment of n or fewer values.
// A NaN in the middle slot is returned unchanged; otherwise the segment around
// the middle is insertion-sorted with a strict < (stable) and its middle read.
CB_HD double window_median_exact(double *v, int n)
{
	int mid = n / 2, a = mid, b = mid;
	if (isnan(v[mid]))
		return v[mid];
	while (a > 0 && !isnan(v[a - 1]))
		--a;
	while (b < n - 1 && !isnan(v[b + 1]))
		++b;
	for (int i = a + 1; i <= b; ++i) {
		double x = v[i];
		int j = i;
		while (j > a && x < v[j - 1]) {
			v[j] = v[j - 1];
			--j;
		}
		v[j] = x;
	}
	return v[mid];
}

} // namespace cb
