"""TEST INFRASTRUCTURE ONLY: pure-Python restatement of GPJSON's JSONPath compiler.

Used by the test suite to cross-check the product compiler (``gpj_compile`` in
the native library) on the reference's golden paths and on random paths.

Follows, line by line:
  gpjson/src/main/java/com/koenv/gpjson/jsonpath/JSONPathParser.java   (grammar, :20-262)
  gpjson/src/main/java/com/koenv/gpjson/jsonpath/JSONPathScanner.java  (cursor, mark/reset stack)
  gpjson/src/main/java/com/koenv/gpjson/jsonpath/IRBuilder.java        (opcode emission, level/store counts)
  gpjson/src/main/java/com/koenv/gpjson/jsonpath/IRByteOutputBuffer.java (LEB128 varints, UTF-8 strings)
  gpjson/src/main/java/com/koenv/gpjson/jsonpath/Opcode.java           (opcode ordinals)

The scanner walks the path as a sequence of Unicode code points, as the Java
scanner walks UTF-16 chars; every character the grammar tests for is ASCII, so
the emitted bytes are identical.
"""

from __future__ import annotations

END, STORE_RESULT, MOVE_UP, MOVE_DOWN, MOVE_TO_KEY, MOVE_TO_INDEX, EXPRESSION_STRING_EQUALS = range(7)

INT_MAX = 2**31 - 1


class JSONPathError(Exception):
    """JSONPathException.java"""


class UnsupportedJSONPathError(JSONPathError):
    """UnsupportedJSONPathException.java"""


class _Scanner:
    """JSONPathScanner.java:3-95"""

    def __init__(self, s: str):
        self.s = s
        self.pos = -1
        self.marks: list[int] = []

    def has_next(self) -> bool:
        return self.pos + 1 < len(self.s)

    def next(self) -> str:
        if not self.has_next():
            raise JSONPathError(f"Expected character, got EOF at {self.pos}")
        self.pos += 1
        return self.s[self.pos]

    def peek(self) -> str:
        if not self.has_next():
            raise JSONPathError(f"Expected character, got EOF at {self.pos}")
        return self.s[self.pos + 1]

    def substring(self, start: int, end: int) -> str:
        return self.s[start + 1:end + 1]

    def expect(self, c: str) -> None:
        got = self.next()
        if got != c:
            raise JSONPathError(f"Expected character '{c}', got character '{got}' at {self.pos}")

    def skip_if(self, c: str) -> bool:
        if not self.has_next():
            return False
        if self.peek() == c:
            self.pos += 1
            return True
        return False

    def error(self, msg: str) -> JSONPathError:
        return JSONPathError(f"{msg} at {self.pos} ('{self.s[self.pos]}')")

    def error_next(self, msg: str) -> JSONPathError:
        return JSONPathError(f"{msg} at {self.pos + 1} ('{self.s[self.pos + 1]}')")

    def unsupported_next(self, msg: str) -> UnsupportedJSONPathError:
        return UnsupportedJSONPathError(f"{msg} at {self.pos + 1} ('{self.s[self.pos + 1]}')")

    def mark(self) -> None:
        self.marks.append(self.pos)

    def reset(self) -> None:
        self.pos = self.marks.pop()


class _IR:
    """IRBuilder.java + IRByteOutputBuffer.java"""

    def __init__(self):
        self.out = bytearray()
        self.level = 0
        self.stores = 0

    def varint(self, i: int) -> None:
        i &= 0xFFFFFFFF
        while i & 0xFFFFFF80:
            self.out.append((i & 0x7F) | 0x80)
            i >>= 7
        self.out.append(i & 0x7F)

    def string(self, s: str) -> None:
        b = s.encode("utf-8", "surrogatepass")
        self.varint(len(b))
        self.out += b

    def prop(self, name: str) -> None:
        self.out.append(MOVE_TO_KEY)
        self.string(name)

    def index(self, i: int) -> None:
        self.out.append(MOVE_TO_INDEX)
        self.varint(i)

    def down(self) -> None:
        self.out.append(MOVE_DOWN)
        self.level += 1

    def up(self) -> None:
        self.out.append(MOVE_UP)
        self.level -= 1

    def store(self) -> None:
        self.out.append(STORE_RESULT)
        self.stores += 1

    def end(self) -> None:
        self.out.append(END)

    def streq(self, s: str) -> None:
        self.out.append(EXPRESSION_STRING_EQUALS)
        self.string('"' + s + '"')


class _Parser:
    """JSONPathParser.java:5-262"""

    def __init__(self, path: str):
        self.sc = _Scanner(path)
        self.ir = _IR()
        self.max_level = 0

    def compile(self):
        self.sc.expect("$")
        self.next_expression()
        self.ir.store()
        self.ir.end()
        return bytes(self.ir.out), self.max_level, self.ir.stores

    def next_expression(self) -> None:
        c = self.sc.peek()
        if c == ".":
            self.dot_expression()
        elif c == "[":
            self.index_expression()
        else:
            raise self.sc.unsupported_next("Unsupported expression type")

    def dot_expression(self) -> None:
        self.sc.expect(".")
        if self.sc.peek() == ".":
            raise self.sc.unsupported_next("Unsupported recursive descent")
        prop = self.read_property()
        if not prop:
            raise self.sc.error("Unexpected empty property")
        self.property_ir(prop)
        if self.sc.has_next():
            self.next_expression()

    def index_expression(self) -> None:
        sc = self.sc
        sc.expect("[")
        p = sc.peek()
        if p in ("'", '"'):
            prop = self.read_quoted()
            if not prop:
                raise sc.error("Unexpected empty property")
            self.property_ir(prop)
        elif "0" <= p <= "9":
            idx = self.read_integer(lambda c: c in "]:,")
            q = sc.peek()
            if q == ":":
                self.range_expression(idx)
                return
            if q == ",":
                raise sc.unsupported_next("Unsupported multiple index expression")
            if q == "]":
                self.index_ir(idx)
        elif p == "*":
            raise sc.unsupported_next("Unsupported wildcard expression")
        elif p == "?":
            self.filter_expression()
        else:
            raise sc.error_next("Unexpected character in index, expected ', \", or an integer")
        sc.expect("]")
        if sc.has_next():
            self.next_expression()

    def range_expression(self, start: int) -> None:
        sc, ir = self.sc, self.ir
        sc.expect(":")
        end = self.read_integer(lambda c: c == "]")
        sc.expect("]")
        max_max = self.max_level
        for i in range(start, end):
            start_level = ir.level
            ir.index(i)
            ir.down()
            sc.mark()
            current_max = self.max_level
            if sc.has_next():
                self.next_expression()
            max_max = max(self.max_level, max_max)
            self.max_level = current_max
            if i == end - 1:
                break
            ir.store()
            sc.reset()
            for _ in range(ir.level - start_level):
                ir.up()
        self.max_level = max_max + 1

    def filter_expression(self) -> None:
        sc = self.sc
        sc.expect("?")
        sc.expect("(")
        sc.expect("@")
        while sc.skip_if(" "):
            pass
        if sc.peek() == "=":
            sc.expect("=")
            sc.expect("=")
            while sc.skip_if(" "):
                pass
            self.ir.streq(self.read_quoted())
        else:
            raise sc.unsupported_next("Unsupported character for expression")
        sc.expect(")")

    def property_ir(self, name: str) -> None:
        self.ir.prop(name)
        self.ir.down()
        self.max_level += 1

    def index_ir(self, i: int) -> None:
        self.ir.index(i)
        self.ir.down()
        self.max_level += 1

    def read_property(self) -> str:
        sc = self.sc
        start = sc.pos
        while sc.has_next():
            c = sc.peek()
            if c == " ":
                raise sc.error_next("Unexpected space")
            if c in ".[":
                break
            sc.next()
        return sc.substring(start, sc.pos)

    def read_quoted(self) -> str:
        sc = self.sc
        q = sc.next()
        if q not in ("'", '"'):
            raise sc.error("Invalid quoted string")
        start = sc.pos
        escaped = False
        while sc.has_next():
            c = sc.peek()
            if escaped:
                escaped = False
            elif c == "\\":
                escaped = True
            elif c == q:
                break
            sc.next()
        end = sc.pos
        sc.expect(q)
        return sc.substring(start, end)

    def read_integer(self, is_end) -> int:
        sc = self.sc
        start = sc.pos
        while sc.has_next():
            c = sc.peek()
            if "0" <= c <= "9":
                sc.next()
                continue
            if is_end(c):
                break
            raise sc.error("Invalid integer")
        text = sc.substring(start, sc.pos)
        # Integer.parseInt: empty or out-of-range text fails to parse.
        if not text or int(text) > INT_MAX:
            raise JSONPathError(f'For input string: "{text}"')
        return int(text)


def compile_path(path: str):
    """Returns (bytecode, max_depth, num_results); raises JSONPathError /
    UnsupportedJSONPathError like JSONPathParser.compile()."""
    return _Parser(path).compile()


def ir_builder():
    """An IRBuilder for writing golden bytecode the way the reference's tests do
    (JSONPathParserTest.java:33-44)."""

    class _B:
        def __init__(self):
            self._ir = _IR()

        def property(self, name):
            self._ir.prop(name)
            return self

        def index(self, i):
            self._ir.index(i)
            return self

        def down(self):
            self._ir.down()
            return self

        def up(self):
            self._ir.up()
            return self

        def storeResult(self):
            self._ir.store()
            return self

        def expressionStringEquals(self, s):
            self._ir.streq(s)
            return self

        def end(self):
            self._ir.end()
            return self

        def toByteArray(self):
            return bytes(self._ir.out)

    return _B()
