// JSONPath subset compiler producing GPJSON bytecode.
//
// Restates gpjson/src/main/java/com/koenv/gpjson/jsonpath/JSONPathParser.java
// (grammar), JSONPathScanner.java (cursor with a mark/reset stack),
// IRBuilder.java and IRByteOutputBuffer.java (encoding), so the bytes are
// identical to the reference compiler's for every input.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace gpj {

// Opcode ordinals (jsonpath/Opcode.java:3-11).
enum Opcode : uint8_t {
    kEnd = 0,
    kStoreResult = 1,
    kMoveUp = 2,
    kMoveDown = 3,
    kMoveToKey = 4,
    kMoveToIndex = 5,
    kExpressionStringEquals = 6,
};

struct CompiledPath {
    std::vector<uint8_t> bytecode;
    int max_depth = 0;    // JSONPathResult.getMaxDepth()
    int num_results = 0;  // JSONPathResult.getNumResults()
};

// JSONPathException / UnsupportedJSONPathException.
struct PathError : std::runtime_error {
    bool unsupported;
    PathError(const std::string& m, bool u) : std::runtime_error(m), unsupported(u) {}
};

// Extensions beyond the reference's subset, off by default (with none set,
// the compiler accepts and rejects exactly what the reference does).
// kPathIndexUnions: `[i,j,...]` with strictly ascending indices, compiled
// like the reference's `[a:b]` ranges (one branch per index: index, down,
// the rest of the path, store, ups back to the array's level), so every
// index keeps its own result slot.  Descending or repeated indices stay
// unsupported: the array's elements are visited once, in order.  As after a
// reference range, an index step later in the path sees the element counter
// of its array carried over from the previous branch.
constexpr unsigned kPathIndexUnions = 1u;

CompiledPath compile_path(const std::string& path, unsigned extensions = 0);

// Static check of bytecode handed to the query kernel: opcodes in range,
// varints of at most 5 bytes with values < 2^31, strings inside the buffer,
// terminated by END, level never below 0 nor above `max_levels`, at most
// `max_stores` STORE_RESULTs.  Fills *depth with the deepest level reached.
bool validate_bytecode(const uint8_t* ir, size_t len, int max_levels, int max_stores,
                       int* depth, int* stores, std::string* why);

}  // namespace gpj
