// JSONPath subset compiler (see jsonpath.h).  Each routine cites the part of
// gpjson/src/main/java/com/koenv/gpjson/jsonpath/JSONPathParser.java it
// restates.  The path is walked as UTF-8 bytes; every character the grammar
// looks at is ASCII, so the emitted bytes equal the reference's.
#include "jsonpath.h"

#include <climits>

namespace gpj {
namespace {

class Cursor {  // JSONPathScanner.java
   public:
    explicit Cursor(const std::string& s) : s_(s) {}

    bool more() const { return pos_ + 1 < static_cast<long>(s_.size()); }
    long pos() const { return pos_; }

    char take() {
        if (!more()) throw PathError("Expected character, got EOF at " + std::to_string(pos_), false);
        return s_[++pos_];
    }
    char look() const {
        if (!more()) throw PathError("Expected character, got EOF at " + std::to_string(pos_), false);
        return s_[pos_ + 1];
    }
    void expect(char c) {
        char got = take();
        if (got != c)
            throw PathError(std::string("Expected character '") + c + "', got character '" + got +
                                "' at " + std::to_string(pos_),
                            false);
    }
    bool skip(char c) {
        if (!more()) return false;
        if (s_[pos_ + 1] != c) return false;
        ++pos_;
        return true;
    }
    std::string slice(long from, long to) const { return s_.substr(from + 1, to - from); }

    PathError error(const std::string& m) const {
        return PathError(m + " at " + std::to_string(pos_) + " ('" + s_[pos_] + "')", false);
    }
    PathError error_next(const std::string& m) const {
        return PathError(m + " at " + std::to_string(pos_ + 1) + " ('" + s_[pos_ + 1] + "')", false);
    }
    PathError unsupported_next(const std::string& m) const {
        return PathError(m + " at " + std::to_string(pos_ + 1) + " ('" + s_[pos_ + 1] + "')", true);
    }

    void push_mark() { marks_.push_back(pos_); }
    void pop_mark() {
        pos_ = marks_.back();
        marks_.pop_back();
    }

   private:
    const std::string& s_;
    long pos_ = -1;
    std::vector<long> marks_;
};

class Emitter {  // IRBuilder.java + IRByteOutputBuffer.java
   public:
    std::vector<uint8_t> out;
    int level = 0;
    int stores = 0;

    void varint(uint32_t v) {  // IRByteOutputBuffer.writeVarInt (:40-47)
        while (v & 0xFFFFFF80u) {
            out.push_back(static_cast<uint8_t>((v & 0x7F) | 0x80));
            v >>= 7;
        }
        out.push_back(static_cast<uint8_t>(v & 0x7F));
    }
    void bytes(const std::string& s) {  // writeString: UTF-8 length + bytes
        varint(static_cast<uint32_t>(s.size()));
        out.insert(out.end(), s.begin(), s.end());
    }
    void key(const std::string& name) { out.push_back(kMoveToKey), bytes(name); }
    void index(int i) { out.push_back(kMoveToIndex), varint(static_cast<uint32_t>(i)); }
    void down() { out.push_back(kMoveDown), ++level; }
    void up() { out.push_back(kMoveUp), --level; }
    void store() { out.push_back(kStoreResult), ++stores; }
    void end() { out.push_back(kEnd); }
    void string_equals(const std::string& s) {
        out.push_back(kExpressionStringEquals);
        bytes("\"" + s + "\"");
    }
};

class Compiler {
   public:
    Compiler(const std::string& path, unsigned extensions) : in_(path), extensions_(extensions) {}

    CompiledPath run() {  // JSONPathParser.compile (:20-29)
        in_.expect('$');
        step();
        ir_.store();
        ir_.end();
        CompiledPath r;
        r.bytecode = std::move(ir_.out);
        r.max_depth = depth_;
        r.num_results = ir_.stores;
        return r;
    }

   private:
    Cursor in_;
    Emitter ir_;
    unsigned extensions_ = 0;
    int depth_ = 0;  // JSONPathParser.maxLevel

    void step() {  // compileNextExpression (:31-43)
        char c = in_.look();
        if (c == '.')
            dot_step();
        else if (c == '[')
            bracket_step();
        else
            throw in_.unsupported_next("Unsupported expression type");
    }

    void dot_step() {  // compileDotExpression (:45-62)
        in_.expect('.');
        if (in_.look() == '.') throw in_.unsupported_next("Unsupported recursive descent");
        std::string name = bare_name();
        if (name.empty()) throw in_.error("Unexpected empty property");
        key_step(name);
        if (in_.more()) step();
    }

    void bracket_step() {  // compileIndexExpression (:64-102)
        in_.expect('[');
        char c = in_.look();
        if (c == '\'' || c == '"') {
            std::string name = quoted();
            if (name.empty()) throw in_.error("Unexpected empty property");
            key_step(name);
        } else if (c >= '0' && c <= '9') {
            int idx = integer(":],");
            char t = in_.look();
            if (t == ':') {
                range_step(idx);  // the range compiles the rest of the path
                return;
            }
            if (t == ',') {
                if (!(extensions_ & kPathIndexUnions))
                    throw in_.unsupported_next("Unsupported multiple index expression");
                union_step(idx);  // like a range, the union compiles the rest of the path
                return;
            }
            if (t == ']') index_step(idx);
        } else if (c == '*') {
            throw in_.unsupported_next("Unsupported wildcard expression");
        } else if (c == '?') {
            filter();
        } else {
            throw in_.error_next("Unexpected character in index, expected ', \", or an integer");
        }
        in_.expect(']');
        if (in_.more()) step();
    }

    // compileIndexRangeExpression (:104-147): one branch per index, each
    // compiling the remainder of the path, joined by STORE_RESULT and enough
    // MOVE_UPs to return to the range's level.
    void range_step(int first) {
        in_.expect(':');
        int last = integer("]");
        in_.expect(']');
        std::vector<int> indices;
        for (int i = first; i < last; i++) indices.push_back(i);
        branches(indices);
    }

    // `[i,j,...]` (kPathIndexUnions): strictly ascending indices, one branch
    // each, as a range.
    void union_step(int first) {
        std::vector<int> indices{first};
        while (in_.skip(',')) {
            while (in_.skip(' ')) {
            }
            const int next = integer(",]");
            if (next <= indices.back()) throw in_.unsupported_next("Unsupported multiple index expression (indices must ascend)");
            indices.push_back(next);
        }
        in_.expect(']');
        branches(indices);
    }

    void branches(const std::vector<int>& indices) {
        int deepest = depth_;
        for (size_t b = 0; b < indices.size(); b++) {
            int base_level = ir_.level;
            ir_.index(indices[b]);
            ir_.down();
            in_.push_mark();
            int saved = depth_;
            if (in_.more()) step();
            if (depth_ > deepest) deepest = depth_;
            depth_ = saved;
            if (b + 1 == indices.size()) break;
            ir_.store();
            in_.pop_mark();
            for (int k = ir_.level - base_level; k > 0; --k) ir_.up();
        }
        depth_ = deepest + 1;
    }

    void filter() {  // compileFilterExpression (:149-177)
        in_.expect('?');
        in_.expect('(');
        in_.expect('@');
        while (in_.skip(' ')) {
        }
        if (in_.look() != '=') throw in_.unsupported_next("Unsupported character for expression");
        in_.expect('=');
        in_.expect('=');
        while (in_.skip(' ')) {
        }
        ir_.string_equals(quoted());
        in_.expect(')');
    }

    void key_step(const std::string& name) {  // createPropertyIR (:179-184)
        ir_.key(name);
        ir_.down();
        ++depth_;
    }
    void index_step(int idx) {  // createIndexIR (:186-191)
        ir_.index(idx);
        ir_.down();
        ++depth_;
    }

    std::string bare_name() {  // readProperty (:193-210)
        long from = in_.pos();
        while (in_.more()) {
            char c = in_.look();
            if (c == ' ') throw in_.error_next("Unexpected space");
            if (c == '.' || c == '[') break;
            in_.take();
        }
        return in_.slice(from, in_.pos());
    }

    std::string quoted() {  // readQuotedString (:212-240): raw text, escapes kept
        char q = in_.take();
        if (q != '\'' && q != '"') throw in_.error("Invalid quoted string");
        long from = in_.pos();
        bool esc = false;
        while (in_.more()) {
            char c = in_.look();
            if (esc)
                esc = false;
            else if (c == '\\')
                esc = true;
            else if (c == q)
                break;
            in_.take();
        }
        long to = in_.pos();
        in_.expect(q);
        return in_.slice(from, to);
    }

    int integer(const char* terminators) {  // readInteger (:242-261) + Integer.parseInt
        long from = in_.pos();
        while (in_.more()) {
            char c = in_.look();
            if (c >= '0' && c <= '9') {
                in_.take();
                continue;
            }
            bool is_end = false;
            for (const char* t = terminators; *t; ++t) is_end |= (c == *t);
            if (is_end) break;
            throw in_.error("Invalid integer");
        }
        std::string digits = in_.slice(from, in_.pos());
        if (digits.empty()) throw PathError("For input string: \"\"", false);
        long long v = 0;
        for (char c : digits) {
            v = v * 10 + (c - '0');
            if (v > INT_MAX) throw PathError("For input string: \"" + digits + "\"", false);
        }
        return static_cast<int>(v);
    }
};

}  // namespace

CompiledPath compile_path(const std::string& path, unsigned extensions) { return Compiler(path, extensions).run(); }

bool validate_bytecode(const uint8_t* ir, size_t len, int max_levels, int max_stores, int* depth,
                       int* stores, std::string* why) {
    size_t pc = 0;
    int level = 0, deepest = 0, n_store = 0;
    auto fail = [&](const char* m) {
        if (why) *why = std::string(m) + " at byte " + std::to_string(pc);
        return false;
    };
    auto varint = [&](uint32_t* v) {
        uint64_t value = 0;
        for (int i = 0; i < 5; i++) {
            if (pc >= len) return false;
            uint8_t b = ir[pc++];
            value |= static_cast<uint64_t>(b & 0x7F) << (7 * i);
            if (!(b & 0x80)) {
                if (value > static_cast<uint64_t>(INT_MAX)) return false;
                *v = static_cast<uint32_t>(value);
                return true;
            }
        }
        return false;
    };
    while (pc < len) {
        uint8_t op = ir[pc++];
        uint32_t v = 0;
        switch (op) {
            case kEnd:
                if (depth) *depth = deepest;
                if (stores) *stores = n_store;
                return true;
            case kStoreResult:
                if (++n_store > max_stores) return fail("more STORE_RESULTs than result slots");
                break;
            case kMoveUp:
                if (--level < 0) return fail("MOVE_UP above level 0");
                break;
            case kMoveDown:
                if (++level > max_levels) return fail("MOVE_DOWN deeper than the index levels");
                if (level > deepest) deepest = level;
                break;
            case kMoveToKey:
            case kExpressionStringEquals:
                // A key search scans the bitmap of the current level, which
                // must exist.
                if (op == kMoveToKey && level >= max_levels)
                    return fail("MOVE_TO_KEY at a level without a bitmap");
                if (!varint(&v)) return fail("bad varint");
                if (v > len - pc) return fail("string runs past the bytecode");
                pc += v;
                break;
            case kMoveToIndex:
                if (level >= max_levels) return fail("MOVE_TO_INDEX at a level without a bitmap");
                if (!varint(&v)) return fail("bad varint");
                break;
            default:
                return fail("unknown opcode");
        }
    }
    return fail("missing END");
}

}  // namespace gpj
