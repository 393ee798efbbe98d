// common.hpp -- shared host-side definitions of the engine: value types, status-carrying errors and
// CUDA call checking.
#pragma once

#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

#include "../../include/vgpu.h"

namespace vgpu {

enum class ValueType : uint8_t {
	INT16 = VGPU_INT16,
	INT32 = VGPU_INT32,
	INT64 = VGPU_INT64,
	FLOAT32 = VGPU_FLOAT32,
	FLOAT64 = VGPU_FLOAT64,
	BOOLEAN = VGPU_BOOLEAN,
	DICTIONARY_STRING = VGPU_DICTIONARY_STRING,
	HUGEINT = VGPU_HUGEINT,
};

inline bool IsValidValueType(uint32_t t) {
	return t <= VGPU_HUGEINT;
}

//! Width of one value in device memory. DICTIONARY_STRING travels as its 32-bit dictionary index.
inline size_t TypeSize(ValueType t) {
	switch (t) {
	case ValueType::INT16:
		return 2;
	case ValueType::INT32:
	case ValueType::FLOAT32:
	case ValueType::DICTIONARY_STRING:
		return 4;
	case ValueType::INT64:
	case ValueType::FLOAT64:
		return 8;
	case ValueType::BOOLEAN:
		return 1;
	case ValueType::HUGEINT:
		return 16;
	}
	return 0;
}

inline bool IsIntegerKeyType(ValueType t) {
	return t == ValueType::INT16 || t == ValueType::INT32 || t == ValueType::INT64 || t == ValueType::BOOLEAN;
}

inline bool IsFloatType(ValueType t) {
	return t == ValueType::FLOAT32 || t == ValueType::FLOAT64;
}

//! C type name the generated kernels use for a value type (the reference translator's CudaTypeName).
inline const char *CudaTypeName(ValueType t) {
	switch (t) {
	case ValueType::INT16:
		return "short";
	case ValueType::INT32:
		return "int";
	case ValueType::INT64:
		return "long long";
	case ValueType::FLOAT32:
		return "float";
	case ValueType::FLOAT64:
		return "double";
	case ValueType::BOOLEAN:
		return "bool";
	case ValueType::DICTIONARY_STRING:
		return "int";
	case ValueType::HUGEINT:
		return "vgpu_dev::u64";
	}
	return "void";
}

inline const char *TypeName(ValueType t) {
	switch (t) {
	case ValueType::INT16:
		return "INT16";
	case ValueType::INT32:
		return "INT32";
	case ValueType::INT64:
		return "INT64";
	case ValueType::FLOAT32:
		return "FLOAT32";
	case ValueType::FLOAT64:
		return "FLOAT64";
	case ValueType::BOOLEAN:
		return "BOOLEAN";
	case ValueType::DICTIONARY_STRING:
		return "DICTIONARY_STRING";
	case ValueType::HUGEINT:
		return "HUGEINT";
	}
	return "?";
}

//! Every engine failure is an Error carrying the status the C ABI returns. Thrown inside the library
//! only; abi.cpp turns it into a status code and a thread-local message.
class Error : public std::runtime_error {
public:
	Error(vgpu_status status, const std::string &message) : std::runtime_error(message), status_(status) {
	}
	vgpu_status status() const {
		return status_;
	}

private:
	vgpu_status status_;
};

[[noreturn]] inline void Fail(vgpu_status status, const std::string &message) {
	throw Error(status, message);
}

inline void CudaCheck(cudaError_t err, const char *what) {
	if (err != cudaSuccess) {
		cudaGetLastError(); // clear a non-sticky error so later calls are not poisoned by it
		vgpu_status status = err == cudaErrorMemoryAllocation ? VGPU_ERR_OUT_OF_MEMORY : VGPU_ERR_CUDA;
		Fail(status, std::string(what) + ": " + cudaGetErrorString(err));
	}
}

#define VGPU_CUDA(call) ::vgpu::CudaCheck((call), #call)

inline uint64_t CeilDiv(uint64_t a, uint64_t b) {
	return (a + b - 1) / b;
}

} // namespace vgpu
