// column_cache.cpp -- see column_cache.hpp. Semantics follow the reference's GpuColumnCache
// (cuda_engine/src/gpu_column_cache.cpp:61-363): staging then commit with a row-count completeness
// gate, byte-budget LRU, whole-table invalidation with a generation counter.
#include "column_cache.hpp"

#include <algorithm>
#include <cstdlib>

#include "kernels.hpp"

namespace vgpu {

ColumnCache &ColumnCache::Get() {
	static ColumnCache *c = new ColumnCache();
	return *c;
}

std::string ColumnCache::TableKey(const TableRef &t) {
	// Length-prefixed components: distinct tables never collide even with dots in identifiers.
	return std::to_string(t.catalog.size()) + ":" + t.catalog + std::to_string(t.schema.size()) + ":" + t.schema +
	       std::to_string(t.table.size()) + ":" + t.table;
}

std::string ColumnCache::Key(const TableRef &t, const std::string &column) {
	return TableKey(t) + std::to_string(column.size()) + ":" + column;
}

void ColumnCache::EnsureInitialized(double fraction) {
	std::lock_guard<std::mutex> lock(mu_);
	if (initialized_) return;
	Runtime::Get().EnsureDevice();
	if (const char *mb = std::getenv("VECTOR_GPU_CACHE_MB")) {
		budget_ = static_cast<uint64_t>(std::atoll(mb)) << 20;
	} else {
		if (const char *f = std::getenv("VECTOR_GPU_CACHE_FRACTION")) {
			double v = std::atof(f);
			if (v >= 0.0 && v <= 1.0) fraction = v;
		}
		size_t free_b = 0, total_b = 0;
		VGPU_CUDA(cudaMemGetInfo(&free_b, &total_b));
		budget_ = static_cast<uint64_t>(static_cast<double>(free_b) * fraction);
	}
	initialized_ = true;
}

void ColumnCache::FreeChunk(Chunk &c) {
	auto &alloc = Runtime::Get().allocator();
	cudaStream_t s = Runtime::Get().default_stream();
	alloc.Free(c.data, s);
	alloc.Free(c.valid, s);
	c.data = nullptr;
	c.valid = nullptr;
}

void ColumnCache::EvictLocked(const std::string &key) {
	auto it = entries_.find(key);
	if (it == entries_.end()) return;
	auto &alloc = Runtime::Get().allocator();
	cudaStream_t s = Runtime::Get().default_stream();
	// Engine executions that read the column may still have kernels queued on their streams: the free is
	// ordered after the marks they left (no device-wide wait). Pointers handed out by GetWhole/TryGetChunk
	// to other code are borrows valid until the next call that can evict, as in the reference's cache.
	it->second.readers->WaitAll(s);
	alloc.Free(it->second.column.data, s);
	alloc.Free(it->second.column.valid, s);
	committed_ -= it->second.bytes;
	lru_.erase(it->second.lru);
	entries_.erase(it);
}

void ColumnCache::EvictTableLocked(const TableRef &table) {
	auto tk = TableKey(table);
	auto it = table_columns_.find(tk);
	if (it == table_columns_.end()) return;
	for (auto &col : it->second) EvictLocked(Key(table, col));
	table_columns_.erase(it);
}

void ColumnCache::AbortLocked(const TableRef &table) {
	auto it = staging_.find(TableKey(table));
	if (it == staging_.end()) return;
	for (auto &kv : it->second) {
		for (auto &c : kv.second.chunks) {
			staged_ -= c.bytes;
			FreeChunk(c);
		}
	}
	staging_.erase(it);
}

bool ColumnCache::MakeRoomLocked(uint64_t bytes) {
	while (committed_ + staged_ + bytes > budget_ && !lru_.empty()) {
		EvictLocked(lru_.back());
	}
	return committed_ + staged_ + bytes <= budget_;
}

void ColumnCache::BeginStaging(const TableRef &table) {
	EnsureInitialized(0.5);
	std::lock_guard<std::mutex> lock(mu_);
	AbortLocked(table);
	// Committed columns of the table stay (as in the reference's cache, gpu_column_cache.cpp:163-172):
	// frequently queried column subsets remain resident; a column staged again replaces its entry at
	// commit, and InvalidateTable drops them all when the table changes.
	if (budget_ == 0) return;
	staging_[TableKey(table)];
}

bool ColumnCache::StageChunk(const TableRef &table, const vgpu_column &chunk) {
	std::lock_guard<std::mutex> lock(mu_);
	auto it = staging_.find(TableKey(table));
	if (it == staging_.end() || chunk.name == nullptr || !IsValidValueType(chunk.type)) return false;
	Staged &st = it->second[chunk.name];
	const ValueType type = static_cast<ValueType>(chunk.type);
	if (st.failed) return false;
	if (st.type_known && st.type != type) {
		st.failed = true;
		for (auto &c : st.chunks) {
			staged_ -= c.bytes;
			FreeChunk(c);
		}
		st.chunks.clear();
		return false;
	}
	const uint64_t bytes = chunk.row_count * TypeSize(type);
	const uint64_t vbytes = chunk.validity ? chunk.row_count : 0;
	if (!MakeRoomLocked(bytes + vbytes)) {
		st.failed = true;
		for (auto &c : st.chunks) {
			staged_ -= c.bytes;
			FreeChunk(c);
		}
		st.chunks.clear();
		return false;
	}
	cudaStream_t s = Runtime::Get().default_stream();
	Chunk c;
	c.rows = chunk.row_count;
	c.bytes = bytes + vbytes;
	c.data = Runtime::Get().allocator().Alloc(bytes, s);
	if (bytes) {
		VGPU_CUDA(cudaMemcpyAsync(c.data, chunk.data, bytes,
		                          chunk.memory == VGPU_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
	}
	if (chunk.validity && chunk.row_count) {
		const size_t vb = (chunk.row_count + 7) / 8;
		uint8_t *bitmap = static_cast<uint8_t *>(Runtime::Get().allocator().Alloc(vb, s));
		VGPU_CUDA(cudaMemcpyAsync(bitmap, chunk.validity, vb,
		                          chunk.memory == VGPU_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
		c.valid = static_cast<uint8_t *>(Runtime::Get().allocator().Alloc(chunk.row_count, s));
		kern::UnpackValidity(bitmap, c.valid, chunk.row_count, s);
		VGPU_CUDA(cudaStreamSynchronize(s));
		Runtime::Get().allocator().Free(bitmap, s);
	}
	VGPU_CUDA(cudaStreamSynchronize(s)); // host source may be reused by the caller after return
	st.type = type;
	st.type_known = true;
	st.rows += c.rows;
	st.bytes += c.bytes;
	staged_ += c.bytes;
	st.chunks.push_back(c);
	return true;
}

bool ColumnCache::StageOwnedChunk(const TableRef &table, const std::string &column, ValueType type, uint64_t rows,
                                  void *data, uint8_t *valid, cudaStream_t stream) {
	std::lock_guard<std::mutex> lock(mu_);
	auto &alloc = Runtime::Get().allocator();
	auto refuse = [&](Staged *st) {
		alloc.Free(data, stream);
		alloc.Free(valid, stream);
		if (st) {
			st->failed = true;
			for (auto &c : st->chunks) {
				staged_ -= c.bytes;
				FreeChunk(c);
			}
			st->chunks.clear();
		}
		return false;
	};
	auto it = staging_.find(TableKey(table));
	if (it == staging_.end()) return refuse(nullptr);
	Staged &st = it->second[column];
	if (st.failed) return refuse(nullptr);
	if (st.type_known && st.type != type) return refuse(&st);
	const uint64_t bytes = rows * TypeSize(type) + (valid ? rows : 0);
	if (!MakeRoomLocked(bytes)) return refuse(&st);
	Chunk c;
	c.data = data;
	c.valid = valid;
	c.rows = rows;
	c.bytes = bytes;
	st.type = type;
	st.type_known = true;
	st.rows += rows;
	st.bytes += bytes;
	staged_ += bytes;
	st.chunks.push_back(c);
	return true;
}

void ColumnCache::CommitStaging(const TableRef &table, uint64_t scanned_rows) {
	std::lock_guard<std::mutex> lock(mu_);
	auto tk = TableKey(table);
	auto it = staging_.find(tk);
	if (it == staging_.end()) return;
	cudaStream_t s = Runtime::Get().default_stream();
	auto &alloc = Runtime::Get().allocator();
	for (auto &kv : it->second) {
		Staged &st = kv.second;
		if (st.failed || st.rows != scanned_rows) {
			for (auto &c : st.chunks) {
				staged_ -= c.bytes;
				FreeChunk(c);
			}
			continue;
		}
		Entry e;
		e.column.name = kv.first;
		e.column.type = st.type;
		e.column.rows = st.rows;
		bool any_valid = false;
		for (auto &c : st.chunks) any_valid |= c.valid != nullptr;
		const size_t w = TypeSize(st.type);
		if (st.chunks.size() == 1 && !any_valid) {
			e.column.data = st.chunks[0].data;
			st.chunks[0].data = nullptr;
		} else {
			e.column.data = alloc.Alloc(st.rows * w, s);
			if (any_valid) e.column.valid = static_cast<uint8_t *>(alloc.Alloc(st.rows, s));
			uint64_t off = 0;
			for (auto &c : st.chunks) {
				if (c.rows) {
					VGPU_CUDA(cudaMemcpyAsync(static_cast<char *>(e.column.data) + off * w, c.data, c.rows * w,
					                          cudaMemcpyDeviceToDevice, s));
					if (any_valid) {
						if (c.valid) {
							VGPU_CUDA(cudaMemcpyAsync(e.column.valid + off, c.valid, c.rows, cudaMemcpyDeviceToDevice, s));
						} else {
							VGPU_CUDA(cudaMemsetAsync(e.column.valid + off, 1, c.rows, s));
						}
					}
				}
				off += c.rows;
			}
		}
		for (auto &c : st.chunks) {
			e.chunk_rows.push_back(c.rows);
			staged_ -= c.bytes;
			FreeChunk(c);
		}
		e.bytes = st.bytes;
		if (IsIntegerKeyType(st.type) || st.type == ValueType::DICTIONARY_STRING) {
			int64_t *mm = static_cast<int64_t *>(alloc.Alloc(16, s));
			kern::MinMaxSigned(e.column.data, static_cast<int>(st.type), st.rows, mm, s);
			int64_t host[2];
			VGPU_CUDA(cudaMemcpyAsync(host, mm, 16, cudaMemcpyDeviceToHost, s));
			VGPU_CUDA(cudaStreamSynchronize(s));
			alloc.Free(mm, s);
			if (st.rows > 0) {
				e.column.has_stats = true;
				e.column.min = host[0];
				e.column.max = host[1];
			}
		}
		const std::string key = Key(table, kv.first);
		const bool replaced = entries_.count(key) != 0;
		if (replaced) EvictLocked(key);  // the column staged again: the new contents replace the old entry
		e.table_key = tk;
		lru_.push_front(key);
		e.lru = lru_.begin();
		committed_ += e.bytes;
		entries_[key] = std::move(e);
		auto &cols = table_columns_[tk];
		if (std::find(cols.begin(), cols.end(), kv.first) == cols.end()) cols.push_back(kv.first);
	}
	VGPU_CUDA(cudaStreamSynchronize(s));
	staging_.erase(it);
	generation_[tk]++;  // new contents: identities taken before no longer match
}

void ColumnCache::AbortStaging(const TableRef &table) {
	std::lock_guard<std::mutex> lock(mu_);
	AbortLocked(table);
}

std::vector<uint64_t> ColumnCache::ReplayableChunkRows(const TableRef &table, const std::vector<std::string> &columns) {
	std::lock_guard<std::mutex> lock(mu_);
	std::vector<uint64_t> rows;
	bool first = true;
	for (auto &c : columns) {
		auto it = entries_.find(Key(table, c));
		if (it == entries_.end()) return {};
		if (first) {
			rows = it->second.chunk_rows;
			first = false;
		} else if (rows != it->second.chunk_rows) {
			return {};
		}
	}
	return rows;
}

bool ColumnCache::TryGetChunk(const TableRef &table, const std::string &column, uint64_t chunk, DevColumn &out) {
	std::lock_guard<std::mutex> lock(mu_);
	auto it = entries_.find(Key(table, column));
	if (it == entries_.end() || chunk >= it->second.chunk_rows.size()) return false;
	lru_.splice(lru_.begin(), lru_, it->second.lru);
	uint64_t off = 0;
	for (uint64_t i = 0; i < chunk; i++) off += it->second.chunk_rows[i];
	const auto &col = it->second.column;
	out = col;
	out.rows = it->second.chunk_rows[chunk];
	out.data = static_cast<char *>(col.data) + off * TypeSize(col.type);
	out.valid = col.valid ? col.valid + off : nullptr;
	out.has_stats = col.has_stats; // the whole-column range bounds every chunk
	return true;
}

bool ColumnCache::GetWhole(const TableRef &table, const std::string &column, DevColumn &out) {
	std::lock_guard<std::mutex> lock(mu_);
	auto it = entries_.find(Key(table, column));
	if (it == entries_.end()) return false;
	lru_.splice(lru_.begin(), lru_, it->second.lru);
	out = it->second.column;
	return true;
}

void ColumnCache::InvalidateTable(const TableRef &table) {
	std::lock_guard<std::mutex> lock(mu_);
	AbortLocked(table);
	EvictTableLocked(table);
	generation_[TableKey(table)]++;
}

void ColumnCache::InvalidateAll() {
	std::lock_guard<std::mutex> lock(mu_);
	while (!lru_.empty()) EvictLocked(lru_.back());
	table_columns_.clear();
	for (auto &kv : staging_) {
		for (auto &col : kv.second) {
			for (auto &c : col.second.chunks) {
				staged_ -= c.bytes;
				FreeChunk(c);
			}
		}
	}
	staging_.clear();
	for (auto &kv : generation_) kv.second++;
}

uint64_t ColumnCache::CurrentBytes() {
	std::lock_guard<std::mutex> lock(mu_);
	return committed_ + staged_;
}

std::string ColumnCache::Identify(const void *data, ValueType type, uint64_t rows) {
	if (data == nullptr) return std::string();
	std::lock_guard<std::mutex> lock(mu_);
	const uint64_t w = TypeSize(type);
	const auto p = reinterpret_cast<uintptr_t>(data);
	for (auto &kv : entries_) {
		const DevColumn &c = kv.second.column;
		if (c.type != type || c.valid) continue;
		const auto base = reinterpret_cast<uintptr_t>(c.data);
		if (p < base || (p - base) % w != 0) continue;
		const uint64_t first = (p - base) / w;
		if (first + rows > c.rows) continue;
		auto g = generation_.find(kv.second.table_key);
		return kv.first + "@" + std::to_string(g == generation_.end() ? 0 : g->second) + "+" + std::to_string(first) +
		       "*" + std::to_string(rows);
	}
	return std::string();
}

bool ColumnCache::BoundsOf(const void *data, ValueType type, uint64_t rows, int64_t *min, int64_t *max) {
	if (data == nullptr || rows == 0) return false;
	std::lock_guard<std::mutex> lock(mu_);
	const uint64_t w = TypeSize(type);
	const auto p = reinterpret_cast<uintptr_t>(data);
	for (auto &kv : entries_) {
		const DevColumn &c = kv.second.column;
		if (c.type != type || !c.has_stats) continue;
		const auto base = reinterpret_cast<uintptr_t>(c.data);
		if (p < base || (p - base) % w != 0 || (p - base) / w + rows > c.rows) continue;
		*min = c.min;
		*max = c.max;
		return true;
	}
	return false;
}

void ColumnCache::AddReaders(const std::vector<const void *> &ptrs, const std::shared_ptr<StreamMark> &mark) {
	if (!mark || ptrs.empty()) return;
	std::lock_guard<std::mutex> lock(mu_);
	for (auto &kv : entries_) {
		const DevColumn &c = kv.second.column;
		const auto base = reinterpret_cast<uintptr_t>(c.data);
		const auto end = base + c.rows * TypeSize(c.type);
		for (const void *p : ptrs) {
			const auto q = reinterpret_cast<uintptr_t>(p);
			if (q >= base && q < end) {
				kv.second.readers->Add(mark);
				break;
			}
		}
	}
}

uint64_t ColumnCache::Generation(const TableRef &table) {
	std::lock_guard<std::mutex> lock(mu_);
	auto it = generation_.find(TableKey(table));
	return it == generation_.end() ? 0 : it->second;
}

} // namespace vgpu
