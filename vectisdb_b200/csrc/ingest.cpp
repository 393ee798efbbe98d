// ingest.cpp -- the host ingest path: DuckDB-shaped chunks -> page-locked batches -> device column cache.
//
// The reference's extension converts each scanned DataChunk on the host (extension/src/vector_converter.cpp:
// 87-273: ToUnifiedFormat, one value per logical row through the selection vector, an Arrow bitmap only
// when a NULL is present), accumulates chunks into pinned batches (gpu_batch_accumulator.cpp:126-249)
// and uploads them with synchronous copies per column chunk (gpu_executor.cu:581-643). Here:
//   - vgpu_convert_vector restates the conversion over a plain description of DuckDB's
//     UnifiedVectorFormat (vgpu_vector: physical data, selection vector, validity words, constant flag),
//     with an optional row selection applied first (the accumulator's `sel` argument);
//   - an ingest handle converts appended chunks straight into one of three page-locked slots of
//     batch_rows rows (values and one valid byte per row), and a full slot is uploaded with
//     asynchronous copies on the handle's own stream into buffers the column cache adopts as staged
//     chunks without copying them again. Filling the next slot overlaps the previous slot's transfer;
//     a slot is refilled only after the event recorded behind its copies has completed.
//   - vgpu_ingest_finish uploads the partial slot, waits for the stream and commits the table, so a
//     query served from the cache sees exactly the appended rows.
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "column_cache.hpp"
#include "runtime.hpp"

namespace vgpu {

namespace {

bool RowValid(const uint64_t *validity, uint64_t phys) {
	return validity == nullptr || ((validity[phys >> 6] >> (phys & 63)) & 1ull) != 0;
}

// The physical index of logical row i of a vector (after the optional row selection).
inline uint64_t Physical(const vgpu_vector &v, const uint32_t *row_sel, uint64_t i) {
	const uint64_t r = row_sel ? row_sel[i] : i;
	if (v.constant) return 0;
	return v.sel ? v.sel[r] : r;
}

// Values of `count` logical rows into `out` (width bytes each) and, when `valid` is given, one byte per
// row (1 = valid). Returns whether a NULL was met.
bool Gather(const vgpu_vector &v, size_t width, uint64_t count, const uint32_t *row_sel, uint8_t *out, uint8_t *valid) {
	bool any_null = false;
	const auto *src = static_cast<const uint8_t *>(v.data);
	switch (width) {
	case 1:
	case 2:
	case 4:
	case 8:
	case 16:
		break;
	default:
		Fail(VGPU_ERR_INVALID_ARGUMENT, "ingest: unsupported value width");
	}
	for (uint64_t i = 0; i < count; i++) {
		const uint64_t p = Physical(v, row_sel, i);
		std::memcpy(out + i * width, src + p * width, width);
		const bool ok = RowValid(v.validity, p);
		any_null |= !ok;
		if (valid) valid[i] = ok ? 1 : 0;
	}
	return any_null;
}

size_t CheckedWidth(uint32_t type) {
	if (!IsValidValueType(type) || static_cast<ValueType>(type) == ValueType::DICTIONARY_STRING) {
		Fail(VGPU_ERR_UNSUPPORTED, "ingest: column type is not a fixed-width numeric type the converter takes");
	}
	return TypeSize(static_cast<ValueType>(type));
}

} // namespace

struct Ingest {
	struct Column {
		std::string name;
		ValueType type;
		size_t width;
	};
	struct Slot {
		std::shared_ptr<uint8_t> host;  // [column values | column valid bytes], page-locked
		cudaEvent_t done = nullptr;     // recorded behind this slot's copies
		bool pending = false;
		std::vector<bool> any_null;
	};
	TableRef table;
	std::vector<Column> cols;
	uint64_t batch_rows = 0;
	uint64_t row_bytes = 0;  // values + one valid byte per column
	std::vector<Slot> slots;
	size_t cur = 0;
	uint64_t fill = 0;
	uint64_t total = 0;
	bool failed = false;
	bool finished = false;
	cudaStream_t stream = nullptr;
	std::mutex mu;

	uint8_t *Values(Slot &s, size_t c) {
		uint64_t off = 0;
		for (size_t i = 0; i < c; i++) off += cols[i].width * batch_rows;
		return s.host.get() + off;
	}
	uint8_t *Valid(Slot &s, size_t c) {
		uint64_t off = 0;
		for (auto &col : cols) off += col.width * batch_rows;
		return s.host.get() + off + c * batch_rows;
	}

	// Uploads the current slot's `fill` rows and hands them to the cache as one staged chunk per column.
	void Flush() {
		if (fill == 0) return;
		Slot &s = slots[cur];
		auto &alloc = Runtime::Get().allocator();
		for (size_t c = 0; c < cols.size(); c++) {
			const uint64_t bytes = fill * cols[c].width;
			void *d = alloc.Alloc(bytes, stream);
			VGPU_CUDA(cudaMemcpyAsync(d, Values(s, c), bytes, cudaMemcpyHostToDevice, stream));
			uint8_t *dv = nullptr;
			if (s.any_null[c]) {
				dv = static_cast<uint8_t *>(alloc.Alloc(fill, stream));
				VGPU_CUDA(cudaMemcpyAsync(dv, Valid(s, c), fill, cudaMemcpyHostToDevice, stream));
			}
			if (!ColumnCache::Get().StageOwnedChunk(table, cols[c].name, cols[c].type, fill, d, dv, stream)) failed = true;
		}
		VGPU_CUDA(cudaEventRecord(s.done, stream));
		s.pending = true;
		total += fill;
		fill = 0;
		cur = (cur + 1) % slots.size();
		Slot &next = slots[cur];
		if (next.pending) {  // the slot about to be refilled: its copies must have left it
			VGPU_CUDA(cudaEventSynchronize(next.done));
			next.pending = false;
		}
		std::fill(next.any_null.begin(), next.any_null.end(), false);
	}

	~Ingest() {
		if (stream) cudaStreamSynchronize(stream);
		if (!finished) {
			try {
				ColumnCache::Get().AbortStaging(table);  // a handle dropped before finishing stages nothing
			} catch (...) {
			}
		}
		for (auto &s : slots) {
			if (s.done) cudaEventDestroy(s.done);
		}
		if (stream) cudaStreamDestroy(stream);
	}
};

} // namespace vgpu

using namespace vgpu;

struct vgpu_ingest {
	std::unique_ptr<Ingest> impl;
};

namespace vgpu {
void SetLastError(const std::string &message);
}

namespace {

template <typename F> vgpu_status IngestGuard(F &&f) {
	try {
		f();
		SetLastError("");
		return VGPU_OK;
	} catch (const Error &e) {
		SetLastError(e.what());
		return e.status();
	} catch (const std::exception &e) {
		SetLastError(e.what());
		return VGPU_ERR_INTERNAL;
	}
}

} // namespace

extern "C" {

vgpu_status vgpu_convert_vector(const vgpu_vector *vector, uint32_t type, uint64_t count, const uint32_t *row_sel,
                                void *out_data, uint8_t *out_validity, int *any_null) {
	return IngestGuard([&] {
		if (!vector || (count && (!vector->data || !out_data))) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		const size_t width = CheckedWidth(type);
		std::vector<uint8_t> valid(out_validity ? count : 0);
		const bool nulls = Gather(*vector, width, count, row_sel, static_cast<uint8_t *>(out_data),
		                          out_validity ? valid.data() : nullptr);
		if (out_validity) {  // Arrow LSB-first, bit set = valid
			std::memset(out_validity, 0, (count + 7) / 8);
			for (uint64_t i = 0; i < count; i++) out_validity[i / 8] |= static_cast<uint8_t>(valid[i] << (i % 8));
		}
		if (any_null) *any_null = nulls ? 1 : 0;
	});
}

vgpu_status vgpu_ingest_create(const vgpu_table_ref *table, const char *const *names, const int32_t *types,
                               size_t n_columns, uint64_t batch_rows, vgpu_ingest **out) {
	return IngestGuard([&] {
		if (!table || !table->table || !out || (n_columns && (!names || !types)) || n_columns == 0) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "ingest: table, columns and output handle are required");
		}
		if (batch_rows == 0 || batch_rows > (1ull << 26)) Fail(VGPU_ERR_INVALID_ARGUMENT, "ingest: batch_rows outside [1, 2^26]");
		Runtime::Get().EnsureDevice();
		auto in = std::make_unique<Ingest>();
		in->table.catalog = table->catalog ? table->catalog : "";
		in->table.schema = table->schema ? table->schema : "";
		in->table.table = table->table;
		for (size_t c = 0; c < n_columns; c++) {
			if (!names[c]) Fail(VGPU_ERR_INVALID_ARGUMENT, "ingest: unnamed column");
			const size_t w = CheckedWidth(static_cast<uint32_t>(types[c]));
			in->cols.push_back({names[c], static_cast<ValueType>(types[c]), w});
			in->row_bytes += w + 1;
		}
		in->batch_rows = batch_rows;
		VGPU_CUDA(cudaStreamCreateWithFlags(&in->stream, cudaStreamNonBlocking));
		in->slots.resize(3);
		for (auto &s : in->slots) {
			s.host = PinnedPool::Get().Acquire(in->row_bytes * batch_rows);
			VGPU_CUDA(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
			s.any_null.assign(n_columns, false);
		}
		ColumnCache::Get().BeginStaging(in->table);
		auto *h = new vgpu_ingest();
		h->impl = std::move(in);
		*out = h;
	});
}

vgpu_status vgpu_ingest_append(vgpu_ingest *h, const vgpu_vector *vectors, uint64_t count, const uint32_t *row_sel) {
	return IngestGuard([&] {
		if (!h || (count && !vectors)) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		Ingest &in = *h->impl;
		std::lock_guard<std::mutex> lock(in.mu);
		if (in.finished) Fail(VGPU_ERR_INVALID_ARGUMENT, "ingest: already finished");
		uint64_t done = 0;
		while (done < count) {  // a chunk larger than the slot's room continues in the next slot
			const uint64_t take = std::min(count - done, in.batch_rows - in.fill);
			Ingest::Slot &s = in.slots[in.cur];
			for (size_t c = 0; c < in.cols.size(); c++) {
				const auto &col = in.cols[c];
				const uint32_t *sel = row_sel ? row_sel + done : nullptr;
				vgpu_vector v = vectors[c];
				if (!v.data && take) Fail(VGPU_ERR_INVALID_ARGUMENT, "ingest: vector without data");
				std::vector<uint32_t> shifted;  // rows past the first `done` of an unselected chunk
				if (!sel && done) {
					shifted.resize(take);
					for (uint64_t i = 0; i < take; i++) shifted[i] = static_cast<uint32_t>(done + i);
					sel = shifted.data();
				}
				if (Gather(v, col.width, take, sel, in.Values(s, c) + in.fill * col.width, in.Valid(s, c) + in.fill)) {
					s.any_null[c] = true;
				}
			}
			in.fill += take;
			done += take;
			if (in.fill == in.batch_rows) in.Flush();
		}
	});
}

vgpu_status vgpu_ingest_finish(vgpu_ingest *h, uint64_t *rows) {
	return IngestGuard([&] {
		if (!h) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		Ingest &in = *h->impl;
		std::lock_guard<std::mutex> lock(in.mu);
		if (in.finished) Fail(VGPU_ERR_INVALID_ARGUMENT, "ingest: already finished");
		in.Flush();
		VGPU_CUDA(cudaStreamSynchronize(in.stream));
		for (auto &s : in.slots) s.pending = false;
		in.finished = true;
		if (in.failed) {
			ColumnCache::Get().AbortStaging(in.table);
			Fail(VGPU_ERR_OUT_OF_MEMORY, "ingest: the column cache had no room for the table (staging aborted)");
		}
		ColumnCache::Get().CommitStaging(in.table, in.total);
		if (rows) *rows = in.total;
	});
}

void vgpu_ingest_destroy(vgpu_ingest *h) {
	if (!h) return;
	try {
		delete h;
	} catch (...) {
	}
}

} // extern "C"
