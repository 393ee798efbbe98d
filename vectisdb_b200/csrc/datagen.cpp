// datagen.cpp -- seeded synthetic column generators for the benchmark configurations (host, OpenMP).
//
// Every value is a pure function of (seed, column id, row): a SplitMix64 stream keyed by
// (seed, column), so any row range is reproducible independently and the output does not depend on
// the thread count. Distributions:
//   uniform integers in [lo, hi)  -- Lemire's multiply-shift on the 64-bit draw
//   uniform doubles in [0, 1)     -- top 53 bits of the draw times 2^-53
//   Zipf(s) ranks over 1..N       -- inverse CDF by binary search in a normalised table
//   permutations                  -- Fisher-Yates driven by the same stream
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

inline uint64_t Finalize(uint64_t z) {
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;

inline uint64_t StreamKey(uint64_t seed, uint32_t column) {
	return Finalize(seed * kGamma + 0x632BE59BD9B4E019ull * (static_cast<uint64_t>(column) + 1));
}

inline uint64_t Draw(uint64_t key, uint64_t row) {
	return Finalize(key + (row + 1) * kGamma);
}

inline uint64_t Below(uint64_t r, uint64_t bound) {
	return static_cast<uint64_t>((static_cast<unsigned __int128>(r) * bound) >> 64);
}

inline double Unit(uint64_t r) {
	return static_cast<double>(r >> 11) * (1.0 / 9007199254740992.0);
}

} // namespace

extern "C" {

void vgdg_uniform_i32(uint64_t seed, uint32_t column, uint64_t offset, uint64_t n, int64_t lo, int64_t hi,
                      int32_t *out) {
	const uint64_t key = StreamKey(seed, column);
	const uint64_t span = static_cast<uint64_t>(hi - lo);
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < static_cast<int64_t>(n); i++) {
		out[i] = static_cast<int32_t>(lo + static_cast<int64_t>(Below(Draw(key, offset + i), span)));
	}
}

void vgdg_uniform_i64(uint64_t seed, uint32_t column, uint64_t offset, uint64_t n, int64_t lo, uint64_t span,
                      int64_t *out) {
	const uint64_t key = StreamKey(seed, column);
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < static_cast<int64_t>(n); i++) {
		out[i] = lo + static_cast<int64_t>(Below(Draw(key, offset + i), span));
	}
}

void vgdg_uniform_f64(uint64_t seed, uint32_t column, uint64_t offset, uint64_t n, double *out) {
	const uint64_t key = StreamKey(seed, column);
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < static_cast<int64_t>(n); i++) {
		out[i] = Unit(Draw(key, offset + i));
	}
}

// cdf[i] = P(rank <= i + 1) for Zipf(s) over ranks 1..n; the last entry is exactly 1.
void vgdg_zipf_cdf(uint64_t n, double s, double *cdf) {
	double total = 0.0;
	for (uint64_t r = 1; r <= n; r++) {
		total += std::pow(static_cast<double>(r), -s);
		cdf[r - 1] = total;
	}
	for (uint64_t i = 0; i < n; i++) {
		cdf[i] /= total;
	}
	if (n) cdf[n - 1] = 1.0;
}

// Zipf rank minus one (0-based) per row.
void vgdg_zipf_i64(uint64_t seed, uint32_t column, uint64_t offset, uint64_t n, const double *cdf, uint64_t values,
                   int64_t *out) {
	const uint64_t key = StreamKey(seed, column);
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < static_cast<int64_t>(n); i++) {
		const double u = Unit(Draw(key, offset + i));
		uint64_t idx = static_cast<uint64_t>(std::upper_bound(cdf, cdf + values, u) - cdf);
		if (idx >= values) idx = values - 1;
		out[i] = static_cast<int64_t>(idx);
	}
}

void vgdg_zipf_i32(uint64_t seed, uint32_t column, uint64_t offset, uint64_t n, const double *cdf, uint64_t values,
                   int32_t *out) {
	const uint64_t key = StreamKey(seed, column);
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < static_cast<int64_t>(n); i++) {
		const double u = Unit(Draw(key, offset + i));
		uint64_t idx = static_cast<uint64_t>(std::upper_bound(cdf, cdf + values, u) - cdf);
		if (idx >= values) idx = values - 1;
		out[i] = static_cast<int32_t>(idx);
	}
}

// Fisher-Yates permutation of [0, n) (sequential: each swap depends on the previous ones).
void vgdg_permutation_i64(uint64_t seed, uint32_t column, uint64_t n, int64_t *out) {
	for (uint64_t i = 0; i < n; i++) out[i] = static_cast<int64_t>(i);
	const uint64_t key = StreamKey(seed, column);
	for (uint64_t i = n; i > 1; i--) {
		const uint64_t j = Below(Draw(key, i - 1), i);
		std::swap(out[i - 1], out[j]);
	}
}

// Join probe keys: with probability hit_fraction a build key at a Zipf rank, else a uniform miss in
// [miss_lo, miss_lo + miss_span).
void vgdg_probe_keys_i64(uint64_t seed, uint32_t column, uint64_t offset, uint64_t n, const int64_t *build_keys,
                         const double *cdf, uint64_t build_n, double hit_fraction, int64_t miss_lo, uint64_t miss_span,
                         int64_t *out) {
	const uint64_t key_sel = StreamKey(seed, column);
	const uint64_t key_rank = StreamKey(seed, column + 1000);
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < static_cast<int64_t>(n); i++) {
		const uint64_t r = Draw(key_sel, offset + i);
		if (Unit(r) < hit_fraction) {
			const double u = Unit(Draw(key_rank, offset + i));
			uint64_t idx = static_cast<uint64_t>(std::upper_bound(cdf, cdf + build_n, u) - cdf);
			if (idx >= build_n) idx = build_n - 1;
			out[i] = build_keys[idx];
		} else {
			out[i] = miss_lo + static_cast<int64_t>(Below(Finalize(r ^ 0xA5A5A5A5A5A5A5A5ull), miss_span));
		}
	}
}

// Lower median (element (n-1)/2 of the sorted order).
int64_t vgdg_median_i64(const int64_t *v, uint64_t n) {
	if (n == 0) return 0;
	std::vector<int64_t> copy(v, v + n);
	auto mid = copy.begin() + static_cast<int64_t>((n - 1) / 2);
	std::nth_element(copy.begin(), mid, copy.end());
	return *mid;
}

} // extern "C"
