"""TEST INFRASTRUCTURE ONLY: a pure-Python restatement of GPUE's equation parser.

GPUE turns ``name = expr`` lines of a parameter file into expression trees and
flattens them into ``EqnNode_gpu`` arrays that a device kernel walks.  This
module restates that parser so the tests can check the library's own C++
parser node for node, and evaluate trees independently of the CUDA path.
The product never imports it.

Reference lines (GPUE-group/GPUE):
  parse_eqn            src/dynamic.cu:227-470
  tree_to_array        src/dynamic.cu:472-507
  find_element_num     src/dynamic.cu:509-522
  evaluate_eqn_gpu     src/dynamic.cu:527-603
  parse_param_file     src/dynamic.cu:187-222 (V gets +0.5*mass*(Ax*Ax+Ay*Ay+Az*Az)
                       appended unless it is the last line)

Grammar properties kept on purpose (they are the reference's behaviour):
  * the split is at the FIRST occurrence of '-', then '+', '/', '*', '^' in that
    priority order, so ``a-b-c`` parses as ``a-(b-c)``;
  * literals are digits and '.' only (no exponent, no unary minus);
  * functions with op number >= 6 keep only their first argument when the tree
    is flattened, so ``jn(a,b)`` evaluates ``jn(a, 0)``;
  * ``pow`` truncates its exponent to int.
"""

import math

MOPS = ["-", "+", "/", "*", "^"]
MOP_NUM = {"+": 1, "-": 2, "*": 3, "/": 4, "^": 5}
FUNC_NUM = {"cos": 6, "sin": 7, "tan": 8, "sqrt": 9, "exp": 10, "pow": 5,
            "jn": 11, "yn": 12, "k2n": 13}


class ParseError(ValueError):
    pass


class Node:
    __slots__ = ("val", "is_dynamic", "var", "left", "right", "op_num", "has_op")

    def __init__(self):
        self.val = 0.0
        self.is_dynamic = False
        self.var = "0"
        self.left = None
        self.right = None
        self.op_num = 0
        self.has_op = False

    def copy(self):
        n = Node()
        n.val, n.is_dynamic, n.var = self.val, self.is_dynamic, self.var
        n.op_num, n.has_op = self.op_num, self.has_op
        n.left = self.left.copy() if self.left is not None else None
        n.right = self.right.copy() if self.right is not None else None
        return n


def parse_eqn(s, doubles, asts, flags=None, name=""):
    """Parse ``s`` (whitespace already removed) into a Node tree.

    doubles: name -> float (GPUE's Grid doubles); asts: name -> Node (earlier
    parameter-file entries).  flags collects names marked time-dependent.
    """
    if flags is None:
        flags = set()
    if len(s) == 0:
        raise ParseError("empty expression")
    ignored = []
    stack = []
    for i, ch in enumerate(s):
        if ch in "([":
            stack.append(i)
        if ch in "])":
            if not stack:
                raise ParseError("unbalanced bracket")
            ignored.append(stack.pop())
            ignored.append(i)
    temp = s
    if ignored:
        if ignored[-1] == len(temp) - 1 and ignored[-2] == 0:
            ignored = ignored[:-2]
            s = s[1:-1]
            ignored = [p - 1 for p in ignored]
        temp = s
        tp = list(ignored)
        for i in range(0, len(tp), 2):
            a, b = tp[i], tp[i + 1]
            temp = temp[:a] + temp[b + 1:]
            for j in range(i + 2, len(tp)):
                if tp[j] > tp[i]:
                    tp[j] -= b - a + 1
    node = Node()
    if all(c in "0123456789." for c in temp):
        node.val = _atof(temp)
        return node
    if len(temp) == 1 and temp in "xyzt":
        node.is_dynamic = True
        node.var = temp
        if temp == "t":
            flags.add(name)
        return node
    mop_point = -1
    for mop in MOPS:
        k = temp.find(mop)
        if k >= 0:
            mop_point = k
            break
    if mop_point < 0:
        if temp in FUNC_NUM:
            mp = len(temp) - 1
            check = s[mp + 1:]
            node.op_num = FUNC_NUM[temp]
            node.has_op = True
            c = check.find(",")
            if c >= 0:
                node.left = parse_eqn(check[1:c], doubles, asts, flags, name)
                node.right = parse_eqn(check[c + 1:len(check) - 1], doubles, asts, flags, name)
            else:
                node.left = parse_eqn(check, doubles, asts, flags, name)
            return node
        if temp in asts:
            flags.add(name)
            return asts[temp].copy()
        if temp in doubles:
            node.val = float(doubles[temp])
            return node
        raise ParseError("No value %s found" % temp)
    if ignored:
        count = 0
        for _ in range(mop_point + 1):
            for j in range(0, len(ignored), 2):
                if ignored[j] == count:
                    count += ignored[j + 1] - ignored[j] + 1
            count += 1
        mop_point = count - 1
    node.op_num = MOP_NUM[s[mop_point]]
    node.has_op = True
    node.left = parse_eqn(s[:mop_point], doubles, asts, flags, name)
    node.right = parse_eqn(s[mop_point + 1:], doubles, asts, flags, name)
    return node


def _atof(t):
    """C atof on a digits-and-dots string: longest valid prefix, else 0."""
    best = 0.0
    for end in range(len(t), 0, -1):
        try:
            best = float(t[:end])
            break
        except ValueError:
            continue
    return best


def tree_to_array(root):
    """Flatten to a list of (val, is_dynamic, var, left, right, op_num)."""
    out = []

    def rec(n):
        idx = len(out)
        out.append([n.val, int(n.is_dynamic), ord(n.var), -1, -1, n.op_num])
        if not n.has_op:
            return
        out[idx][3] = len(out)
        rec(n.left)
        if n.op_num < 6:
            out[idx][4] = len(out)
            rec(n.right)

    rec(root)
    return out


def _factorial(v):
    r = v
    if v < 1:
        return 1.0
    for i in range(int(math.floor(v)) - 1, 0, -1):
        r *= i
    return r


def _cpow(a, b):
    r = math.sqrt(a.real * a.real + a.imag * a.imag)
    th = math.atan(a.imag / a.real) if a.real != 0 else math.copysign(math.pi / 2, a.imag)
    return complex(r ** b * math.cos(b * th), r ** b * math.sin(b * th))


def _poly_i(v, x, n):
    ival = 0j
    x = 1j * x
    for i in range(n):
        b = (-1.0) ** i * (_factorial(n + i - 1) * float(n) ** (1 - 2 * i)) / (
            _factorial(i) * _factorial(n - i) * _factorial(v + i))
        ival += _cpow(x * 0.5, 2 * i + v) * b
    return ival


def evaluate(arr, x, y, z, t, k=0):
    """evaluate_eqn_gpu on a flattened array (Python floats)."""
    val, dyn, var, left, right, op = arr[k]
    if right < 0 and left < 0:
        if dyn:
            return {ord("x"): x, ord("y"): y, ord("z"): z, ord("t"): t}[var]
        return val
    a = evaluate(arr, x, y, z, t, left) if left > 0 else 0.0
    b = evaluate(arr, x, y, z, t, right) if right > 0 else 0.0
    if op == 1:
        return a + b
    if op == 2:
        return a - b
    if op == 3:
        return a * b
    if op == 4:
        return a / b if b != 0 else math.copysign(math.inf, a) if a != 0 else math.nan
    if op == 5:
        return math.pow(a, int(b))
    if op == 6:
        return math.cos(a)
    if op == 7:
        return math.sin(a)
    if op == 8:
        return math.tan(a)
    if op == 9:
        return math.sqrt(a)
    if op == 10:
        return math.exp(a)
    if op in (11, 12):
        import scipy.special as sp
        n = int(a)
        return float(sp.jv(n, b)) if op == 11 else float(sp.yv(n, b))
    if op == 13:
        v = int(a)
        n = 30
        val = (_poly_i(-v, complex(b, 0), n) - _poly_i(v, complex(b, 0), n)) * (
            math.pi / (2 * math.sin(n * math.pi)))
        return (val * val).real
    return 0.0


def parse_param_text(text, doubles):
    """parse_param_file on the text of a parameter file.

    Returns (asts: name -> Node, order: [names], time_flags: set)."""
    asts, order, flags = {}, [], set()
    val_string, eqn_string = "", ""

    def allocate(name, expr):
        asts[name] = parse_eqn(expr, doubles, asts, flags, name)
        if name not in order:
            order.append(name)

    for line in text.splitlines():
        line = "".join(ch for ch in line if not ch.isspace())
        it = line.find("=")
        if it < 0:
            eqn_string += line
        else:
            if val_string != "":
                if val_string == "V":
                    eqn_string += "+0.5*mass*(Ax*Ax+Ay*Ay+Az*Az)"
                allocate(val_string, eqn_string)
                val_string, eqn_string = "", ""
            val_string = line[:it]
            eqn_string = line[it + 1:]
    allocate(val_string, eqn_string)
    return asts, order, flags
