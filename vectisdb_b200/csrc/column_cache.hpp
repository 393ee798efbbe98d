// column_cache.hpp -- device-resident column cache: the reference's GpuColumnCache
// (cuda_engine/include/gpu_column_cache.hpp:107-281, src/gpu_column_cache.cpp) re-built for a
// resident-column B200: committed columns are ONE contiguous device buffer each (chunk boundaries are
// kept as offsets, so chunk replay is a pointer offset and whole-column serving is zero-copy), and the
// integer range of every column is computed once at commit so group-by key packing needs no pass.
#pragma once

#include <list>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "executor.hpp"
#include "plan.hpp"

namespace vgpu {

class ColumnCache {
public:
	static ColumnCache &Get();

	void EnsureInitialized(double fraction_of_vram);
	void BeginStaging(const TableRef &table);
	bool StageChunk(const TableRef &table, const vgpu_column &chunk);
	//! Stages a chunk whose device buffers the caller allocated from the engine's allocator and filled
	//! with work on `stream`: the cache takes ownership without copying (data: rows values of `type`;
	//! valid: one byte per row, 1 = valid, or nullptr). The caller synchronizes `stream` before the
	//! commit. False (buffers freed on `stream`) when the slot is closed, the type changed or the
	//! budget has no room.
	bool StageOwnedChunk(const TableRef &table, const std::string &column, ValueType type, uint64_t rows, void *data,
	                     uint8_t *valid, cudaStream_t stream);
	void CommitStaging(const TableRef &table, uint64_t scanned_rows);
	void AbortStaging(const TableRef &table);
	std::vector<uint64_t> ReplayableChunkRows(const TableRef &table, const std::vector<std::string> &columns);
	bool TryGetChunk(const TableRef &table, const std::string &column, uint64_t chunk, DevColumn &out);
	//! Borrow of the whole committed column (zero-copy); false on a miss.
	bool GetWhole(const TableRef &table, const std::string &column, DevColumn &out);
	void InvalidateTable(const TableRef &table);
	void InvalidateAll();
	uint64_t CurrentBytes();
	uint64_t Generation(const TableRef &table);
	//! Identity of cache-owned device data: "(table, column)@generation+offset*rows" when `rows`
	//! values of `type` at `data` lie inside one committed column, else "". Contents behind an identity
	//! never change (re-staging or invalidating a table bumps its generation), so derived structures
	//! keyed by it (join tables) stay valid.
	std::string Identify(const void *data, ValueType type, uint64_t rows);
	//! The committed column's value range when `rows` values at `data` lie inside one (a superset of
	//! those rows' range, valid for key packing); false otherwise.
	bool BoundsOf(const void *data, ValueType type, uint64_t rows, int64_t *min, int64_t *max);
	//! Records `mark` (after an execution's last kernel) on every committed column that one of `ptrs`
	//! points into: evicting such a column frees its buffers only after the marked work. Pointers
	//! outside the cache are ignored.
	void AddReaders(const std::vector<const void *> &ptrs, const std::shared_ptr<StreamMark> &mark);

private:
	struct Chunk {
		void *data = nullptr;
		uint8_t *valid = nullptr;
		uint64_t rows = 0;
		uint64_t bytes = 0;
	};
	struct Staged {
		std::vector<Chunk> chunks;
		ValueType type = ValueType::INT32;
		bool type_known = false;
		bool failed = false;
		uint64_t rows = 0;
		uint64_t bytes = 0;
	};
	struct Entry {
		DevColumn column; // contiguous data (+ byte validity), stats filled
		std::string table_key;
		std::vector<uint64_t> chunk_rows;
		uint64_t bytes = 0;
		std::list<std::string>::iterator lru;
		std::shared_ptr<ReaderMarks> readers = std::make_shared<ReaderMarks>();  // engine executions that read it
	};
	static std::string Key(const TableRef &t, const std::string &column);
	static std::string TableKey(const TableRef &t);
	void EvictLocked(const std::string &key);
	void EvictTableLocked(const TableRef &table);
	void AbortLocked(const TableRef &table);
	void FreeChunk(Chunk &c);
	bool MakeRoomLocked(uint64_t bytes);

	std::mutex mu_;
	bool initialized_ = false;
	uint64_t budget_ = 0;
	uint64_t committed_ = 0;
	uint64_t staged_ = 0;
	std::list<std::string> lru_;
	std::unordered_map<std::string, Entry> entries_;
	std::unordered_map<std::string, std::unordered_map<std::string, Staged>> staging_;
	std::unordered_map<std::string, std::vector<std::string>> table_columns_;
	std::unordered_map<std::string, uint64_t> generation_;
};

} // namespace vgpu
