// oracle.cpp -- CPU restatement of the benchmark queries, used ONLY as the parity checker in tests/,
// smoke() and the CPU-baseline leg of bench.py. Never linked into, or called by, the product path.
//
// Each function restates DuckDB's semantics for one query over host arrays, multithreaded with
// OpenMP the way DuckDB's CPU operators are (radix-partitioned hash aggregation, a hash/sort join):
//   - GROUP BY output is an unordered set; results are returned sorted by key for comparison.
//   - COUNT(*) -> BIGINT; MIN/MAX keep the input type; SUM over BIGINT/DECIMAL(18,2) is exact and
//     128-bit (DECIMAL(38,2)); SUM/AVG over DOUBLE accumulate in double (order-dependent, compared
//     within 1e-12 relative); BIGINT % truncates toward zero (C semantics).
//   - INNER equi-join emits each matching (left, right) pair once (a build key repeated r times pairs
//     every matching probe row r times); cross product is left-major.
// Built with -ffp-contract=off so v*2+1 rounds twice, as DuckDB (and the engine, --fmad=false) do.
//
// Reference anchors: the aggregate rules follow cuda_engine/src/operators/gpu_groupby.cu:24-37 and
// extension/src/expression_translator.cpp:65-101, 428-438; the join output contract follows
// cuda_engine/src/operators/gpu_hash_join.cu:25-38; the cross-product order follows
// cuda_engine/src/operators/gpu_cross_join.cu:16-19.
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

struct C0State {
	double sum = 0.0;
	int64_t cnt = 0;
	int64_t mn = INT64_MAX, mx = INT64_MIN;
};

struct C1State {
	__int128 amt = 0;
	double vsum = 0.0;
	int64_t cnt = 0;
	int64_t mx = INT64_MIN;
};

inline uint64_t Mix(uint64_t k) {
	k ^= k >> 33;
	k *= 0xff51afd7ed558ccdull;
	k ^= k >> 33;
	k *= 0xc4ceb9fe1a85ec53ull;
	k ^= k >> 33;
	return k;
}

} // namespace

extern "C" {

int oracle_threads(void) {
	return omp_get_max_threads();
}

void oracle_set_threads(int n) {
	if (n > 0) omp_set_num_threads(n);
}

// SELECT k, SUM(v*2+1), COUNT(*), MIN(w), MAX(w) FROM t WHERE v < v_lt AND w % w_mod <> 0 GROUP BY k
// Outputs sorted by k; returns the group count (capacity must be >= the number of distinct k).
int64_t oracle_c0(const int32_t *k, const double *v, const int64_t *w, uint64_t n, double v_lt, int64_t w_mod,
                  int32_t *out_k, double *out_sum, int64_t *out_cnt, int64_t *out_min, int64_t *out_max,
                  uint64_t capacity) {
	const int T = omp_get_max_threads();
	std::vector<std::unordered_map<int32_t, C0State>> partial(T);
#pragma omp parallel
	{
		auto &m = partial[omp_get_thread_num()];
#pragma omp for schedule(static)
		for (int64_t i = 0; i < static_cast<int64_t>(n); i++) {
			if (v[i] < v_lt && (w[i] % w_mod) != 0) {
				auto &s = m[k[i]];
				const double x = v[i] * 2.0 + 1.0;
				s.sum += x;
				s.cnt += 1;
				s.mn = std::min(s.mn, w[i]);
				s.mx = std::max(s.mx, w[i]);
			}
		}
	}
	std::unordered_map<int32_t, C0State> merged;
	for (auto &m : partial) {
		for (auto &kv : m) {
			auto &s = merged[kv.first];
			s.sum += kv.second.sum;
			s.cnt += kv.second.cnt;
			s.mn = std::min(s.mn, kv.second.mn);
			s.mx = std::max(s.mx, kv.second.mx);
		}
	}
	std::vector<int32_t> keys;
	for (auto &kv : merged) keys.push_back(kv.first);
	std::sort(keys.begin(), keys.end());
	if (keys.size() > capacity) return -1;
	for (size_t i = 0; i < keys.size(); i++) {
		const auto &s = merged[keys[i]];
		out_k[i] = keys[i];
		out_sum[i] = s.sum;
		out_cnt[i] = s.cnt;
		out_min[i] = s.mn;
		out_max[i] = s.mx;
	}
	return static_cast<int64_t>(keys.size());
}

// SELECT k, v*2+1, w FROM t WHERE v < v_lt AND w % w_mod <> 0 -- the filter and projection alone,
// passing rows in input order (the reference's stable compaction, gpu_executor.cu:645-746).
// Pass out_k == nullptr to only count. Returns the passing row count.
int64_t oracle_cp(const int32_t *k, const double *v, const int64_t *w, uint64_t n, double v_lt, int64_t w_mod,
                  int32_t *out_k, double *out_v, int64_t *out_w, uint64_t capacity) {
	const int T = omp_get_max_threads();
	std::vector<uint64_t> start(static_cast<size_t>(T) + 1, 0);
#pragma omp parallel
	{
		const int t = omp_get_thread_num();
		const uint64_t lo = n * t / T, hi = n * (t + 1) / T;
		uint64_t c = 0;
		for (uint64_t i = lo; i < hi; i++) c += (v[i] < v_lt && (w[i] % w_mod) != 0);
		start[t + 1] = c;
#pragma omp barrier
#pragma omp single
		for (int j = 0; j < T; j++) start[j + 1] += start[j];
		if (out_k != nullptr && start[T] <= capacity) {
			uint64_t pos = start[t];
			for (uint64_t i = lo; i < hi; i++) {
				if (v[i] < v_lt && (w[i] % w_mod) != 0) {
					out_k[pos] = k[i];
					out_v[pos] = v[i] * 2.0 + 1.0;
					out_w[pos] = w[i];
					pos++;
				}
			}
		}
	}
	if (out_k != nullptr && start[T] > capacity) return -1;
	return static_cast<int64_t>(start[T]);
}

// SELECT a, b, SUM(amt), AVG(v), COUNT(*), MAX(ts) FROM t WHERE ts > ts_gt GROUP BY a, b
// Radix-partitioned hash aggregation. Outputs sorted by (a, b); SUM(amt) as (lower, upper) halves.
int64_t oracle_c1(const int32_t *a, const int32_t *b, const int64_t *amt, const double *v, const int64_t *ts,
                  uint64_t n, int64_t ts_gt, int32_t *out_a, int32_t *out_b, uint64_t *out_sum_lo, int64_t *out_sum_hi,
                  double *out_avg, int64_t *out_cnt, int64_t *out_max, uint64_t capacity) {
	const int T = omp_get_max_threads();
	constexpr int P = 256;
	std::vector<std::vector<uint64_t>> counts(T, std::vector<uint64_t>(P, 0));
	// phase 1a: count qualifying rows per (thread, partition)
#pragma omp parallel
	{
		const int t = omp_get_thread_num();
		auto &c = counts[t];
#pragma omp for schedule(static)
		for (int64_t i = 0; i < static_cast<int64_t>(n); i++) {
			if (ts[i] > ts_gt) {
				const uint64_t key = (static_cast<uint64_t>(static_cast<uint32_t>(a[i])) << 32) | static_cast<uint32_t>(b[i]);
				c[Mix(key) >> 56]++;
			}
		}
	}
	std::vector<uint64_t> offset(static_cast<size_t>(P) * T);
	uint64_t total = 0;
	for (int p = 0; p < P; p++) {
		for (int t = 0; t < T; t++) {
			offset[static_cast<size_t>(p) * T + t] = total;
			total += counts[t][p];
		}
	}
	std::vector<uint64_t> pkey(total);
	std::vector<uint64_t> prow(total);
	// phase 1b: scatter (key, row) into partition-major order (same static schedule as 1a)
#pragma omp parallel
	{
		const int t = omp_get_thread_num();
		std::vector<uint64_t> cur(P);
		for (int p = 0; p < P; p++) cur[p] = offset[static_cast<size_t>(p) * T + t];
#pragma omp for schedule(static)
		for (int64_t i = 0; i < static_cast<int64_t>(n); i++) {
			if (ts[i] > ts_gt) {
				const uint64_t key = (static_cast<uint64_t>(static_cast<uint32_t>(a[i])) << 32) | static_cast<uint32_t>(b[i]);
				const uint64_t pos = cur[Mix(key) >> 56]++;
				pkey[pos] = key;
				prow[pos] = static_cast<uint64_t>(i);
			}
		}
	}
	// phase 2: aggregate each partition independently
	std::vector<std::vector<std::pair<uint64_t, C1State>>> groups(P);
#pragma omp parallel for schedule(dynamic, 1)
	for (int p = 0; p < P; p++) {
		const uint64_t start = offset[static_cast<size_t>(p) * T];
		const uint64_t end = p + 1 < P ? offset[static_cast<size_t>(p + 1) * T] : total;
		std::unordered_map<uint64_t, C1State> m;
		m.reserve((end - start) / 2 + 16);
		for (uint64_t j = start; j < end; j++) {
			const uint64_t i = prow[j];
			auto &s = m[pkey[j]];
			s.amt += amt[i];
			s.vsum += v[i];
			s.cnt += 1;
			s.mx = std::max(s.mx, ts[i]);
		}
		auto &g = groups[p];
		g.reserve(m.size());
		for (auto &kv : m) g.push_back(kv);
	}
	std::vector<std::pair<uint64_t, C1State>> all;
	for (auto &g : groups) all.insert(all.end(), g.begin(), g.end());
	if (all.size() > capacity) return -1;
	std::sort(all.begin(), all.end(), [](const auto &x, const auto &y) {
		const int32_t ax = static_cast<int32_t>(x.first >> 32), ay = static_cast<int32_t>(y.first >> 32);
		if (ax != ay) return ax < ay;
		return static_cast<int32_t>(x.first & 0xffffffffu) < static_cast<int32_t>(y.first & 0xffffffffu);
	});
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < static_cast<int64_t>(all.size()); i++) {
		const auto &s = all[i].second;
		out_a[i] = static_cast<int32_t>(all[i].first >> 32);
		out_b[i] = static_cast<int32_t>(all[i].first & 0xffffffffu);
		out_sum_lo[i] = static_cast<uint64_t>(s.amt);
		out_sum_hi[i] = static_cast<int64_t>(s.amt >> 64);
		out_avg[i] = s.vsum / static_cast<double>(s.cnt);
		out_cnt[i] = s.cnt;
		out_max[i] = s.mx;
	}
	return static_cast<int64_t>(all.size());
}

// SELECT b.g, SUM(p.x), COUNT(*) FROM probe p JOIN build b ON p.key = b.key GROUP BY b.g
// A hash join, as DuckDB's CPU plan runs it: the build side goes into an open-addressing table (linear
// probing, duplicate keys kept as separate entries), each probe row walks its run of the table and
// emits one pair per equal key, so a build key that repeats r times counts the probe row r times.
// Per-thread partial aggregates in row order, merged in thread order. Outputs sorted by g.
int64_t oracle_c2(const int64_t *bkey, const int32_t *bg, uint64_t bn, const int64_t *pkey, const double *px,
                  uint64_t pn, int32_t *out_g, double *out_sum, int64_t *out_cnt, uint64_t capacity) {
	uint64_t slots = 16;
	while (slots < 2 * bn) slots <<= 1;
	const uint64_t mask = slots - 1;
	std::vector<int64_t> tkey(slots);
	std::vector<int32_t> tg(slots);
	std::vector<uint8_t> used(slots, 0);
	for (uint64_t i = 0; i < bn; i++) {
		uint64_t h = Mix(static_cast<uint64_t>(bkey[i])) & mask;
		while (used[h]) h = (h + 1) & mask;
		used[h] = 1;
		tkey[h] = bkey[i];
		tg[h] = bg[i];
	}
	int32_t gmin = INT32_MAX, gmax = INT32_MIN;
	for (uint64_t i = 0; i < bn; i++) {
		gmin = std::min(gmin, bg[i]);
		gmax = std::max(gmax, bg[i]);
	}
	const int T = omp_get_max_threads();
	const bool dense = bn > 0 && static_cast<int64_t>(gmax) - gmin < (1 << 20);
	const uint64_t G = dense ? static_cast<uint64_t>(static_cast<int64_t>(gmax) - gmin + 1) : 0;
	std::vector<std::vector<double>> dsum(T, std::vector<double>(G, 0.0));
	std::vector<std::vector<int64_t>> dcnt(T, std::vector<int64_t>(G, 0));
	std::vector<std::unordered_map<int32_t, std::pair<double, int64_t>>> partial(T);
#pragma omp parallel
	{
		const int t = omp_get_thread_num();
		auto &m = partial[t];
		auto &ds = dsum[t];
		auto &dc = dcnt[t];
#pragma omp for schedule(static)
		for (int64_t i = 0; i < static_cast<int64_t>(pn); i++) {
			const int64_t key = pkey[i];
			for (uint64_t h = Mix(static_cast<uint64_t>(key)) & mask; used[h]; h = (h + 1) & mask) {
				if (tkey[h] != key) continue;
				if (dense) {
					ds[tg[h] - gmin] += px[i];
					dc[tg[h] - gmin] += 1;
				} else {
					auto &st = m[tg[h]];
					st.first += px[i];
					st.second += 1;
				}
			}
		}
	}
	std::unordered_map<int32_t, std::pair<double, int64_t>> merged;
	for (int t = 0; t < T; t++) {
		for (uint64_t j = 0; j < G; j++) {
			if (dcnt[t][j] == 0) continue;
			auto &st = merged[static_cast<int32_t>(gmin + static_cast<int64_t>(j))];
			st.first += dsum[t][j];
			st.second += dcnt[t][j];
		}
		for (auto &kv : partial[t]) {
			auto &st = merged[kv.first];
			st.first += kv.second.first;
			st.second += kv.second.second;
		}
	}
	std::vector<int32_t> keys;
	for (auto &kv : merged) keys.push_back(kv.first);
	std::sort(keys.begin(), keys.end());
	if (keys.size() > capacity) return -1;
	for (size_t i = 0; i < keys.size(); i++) {
		out_g[i] = keys[i];
		out_sum[i] = merged[keys[i]].first;
		out_cnt[i] = merged[keys[i]].second;
	}
	return static_cast<int64_t>(keys.size());
}

// SELECT l.a, r.b FROM l, r WHERE (l.a + r.b) % modulus = 0, left-major order.
// Pass out_a == nullptr to only count. Returns the pair count.
int64_t oracle_c2b(const int32_t *la, uint64_t ln, const int32_t *rb, uint64_t rn, int32_t modulus, int32_t *out_a,
                   int32_t *out_b, uint64_t capacity) {
	std::vector<uint64_t> per_left(ln + 1, 0);
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < static_cast<int64_t>(ln); i++) {
		uint64_t c = 0;
		for (uint64_t j = 0; j < rn; j++) c += ((la[i] + rb[j]) % modulus) == 0;
		per_left[i + 1] = c;
	}
	for (uint64_t i = 0; i < ln; i++) per_left[i + 1] += per_left[i];
	const uint64_t total = per_left[ln];
	if (out_a == nullptr) return static_cast<int64_t>(total);
	if (total > capacity) return -1;
#pragma omp parallel for schedule(static)
	for (int64_t i = 0; i < static_cast<int64_t>(ln); i++) {
		uint64_t pos = per_left[i];
		for (uint64_t j = 0; j < rn; j++) {
			if (((la[i] + rb[j]) % modulus) == 0) {
				out_a[pos] = la[i];
				out_b[pos] = rb[j];
				pos++;
			}
		}
	}
	return static_cast<int64_t>(total);
}

} // extern "C"
