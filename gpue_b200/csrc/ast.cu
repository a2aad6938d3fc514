// ast.cpp -- host side of GPUE's equation strings (see ast.h).
//
// The grammar is GPUE's, quirks included, because parameter files written for
// GPUE must mean the same thing here (parse_eqn, src/dynamic.cu:227-470):
//   * brackets are matched first; a bracket pair around the whole string is
//     dropped; bracketed spans are hidden while looking for an operator;
//   * the split is at the FIRST occurrence of '-', else '+', '/', '*', '^' (in
//     that priority), so "a-b-c" is a-(b-c);
//   * a string of digits and '.' only is a literal (C atof, so "" is 0);
//   * x, y, z, t are variables; cos sin tan sqrt exp pow jn yn k2n are
//     functions, with "name(a,b)" split at the first comma;
//   * any other name is an earlier expression of the file (copied in, and the
//     result marked time dependent) or one of the Grid doubles;
//   * flattening keeps only the first argument of functions numbered >= 6
//     (tree_to_array), so jn(a,b) evaluates jn(a, 0).

#include "ast.h"
#include "ast_eval.cuh"

#include <cctype>
#include <cmath>
#include <cstdlib>
#include <functional>
#include <memory>
#include <stack>

namespace gpue {

namespace {

struct TNode {
    double val = 0.0;
    bool dyn = false;
    char var = '0';
    int op = 0;
    bool has_op = false;
    std::shared_ptr<TNode> l, r;
};

std::shared_ptr<TNode> clone(const std::shared_ptr<TNode>& n) {
    if (!n) return nullptr;
    auto c = std::make_shared<TNode>(*n);
    c->l = clone(n->l);
    c->r = clone(n->r);
    return c;
}

const std::map<std::string, int>& functions() {
    static const std::map<std::string, int> m = {
        {"cos", 6}, {"sin", 7}, {"tan", 8}, {"sqrt", 9}, {"exp", 10},
        {"pow", 5}, {"jn", 11}, {"yn", 12}, {"k2n", 13}};
    return m;
}

int operator_num(char c) {
    switch (c) {
        case '+': return 1;
        case '-': return 2;
        case '*': return 3;
        case '/': return 4;
        case '^': return 5;
        default: return 0;
    }
}

struct Parser {
    const std::map<std::string, double>& doubles;
    const std::map<std::string, std::shared_ptr<TNode>>& trees;
    bool time_dep = false;
    std::string err;
    int depth = 0;

    std::shared_ptr<TNode> parse(std::string s) {
        if (!err.empty()) return nullptr;
        if (s.empty()) {
            err = "empty expression";
            return nullptr;
        }
        if (++depth > 400) {
            err = "expression nested too deeply";
            return nullptr;
        }
        struct Guard {
            int& d;
            ~Guard() { --d; }
        } guard{depth};
        // bracket pairs, recorded when they close
        std::vector<int> ign;
        std::stack<int> open;
        for (int i = 0; i < (int)s.size(); ++i) {
            if (s[i] == '(' || s[i] == '[') open.push(i);
            if (s[i] == ']' || s[i] == ')') {
                if (open.empty()) {
                    err = "unbalanced bracket in '" + s + "'";
                    return nullptr;
                }
                ign.push_back(open.top());
                ign.push_back(i);
                open.pop();
            }
        }
        std::string temp = s;
        if (!ign.empty()) {
            if (ign[ign.size() - 1] == (int)temp.size() - 1 && ign[ign.size() - 2] == 0) {
                ign.pop_back();
                ign.pop_back();
                s = s.substr(1, s.size() - 2);
                for (auto& p : ign) --p;
            }
            temp = s;
            std::vector<int> tp = ign;
            for (size_t i = 0; i < tp.size(); i += 2) {
                const int a = tp[i], b = tp[i + 1];
                temp.erase(a, b - a + 1);
                for (size_t j = i + 2; j < tp.size(); ++j)
                    if (tp[j] > tp[i]) tp[j] -= b - a + 1;
            }
        }
        auto node = std::make_shared<TNode>();
        if (temp.find_first_not_of("0123456789.") == std::string::npos) {
            node->val = std::atof(temp.c_str());
            return node;
        }
        if (temp.size() == 1 &&
            (temp[0] == 'x' || temp[0] == 'y' || temp[0] == 'z' || temp[0] == 't')) {
            node->dyn = true;
            node->var = temp[0];
            if (temp[0] == 't') time_dep = true;
            return node;
        }
        int mop = -1;
        for (const char* m : {"-", "+", "/", "*", "^"}) {
            const size_t k = temp.find(m);
            if (k != std::string::npos) {
                mop = (int)k;
                break;
            }
        }
        if (mop < 0) {
            auto f = functions().find(temp);
            if (f != functions().end()) {
                const int mp = (int)temp.size() - 1;
                const std::string check = s.substr(mp + 1);
                node->op = f->second;
                node->has_op = true;
                const size_t comma = check.find(',');
                if (comma != std::string::npos) {
                    if (check.size() < 2 || comma < 1) {
                        err = "malformed arguments in '" + s + "'";
                        return nullptr;
                    }
                    node->l = parse(check.substr(1, comma - 1));
                    node->r = parse(check.substr(comma + 1, check.size() - comma - 2));
                } else {
                    node->l = parse(check);
                }
                return err.empty() ? node : nullptr;
            }
            auto t = trees.find(temp);
            if (t != trees.end()) {
                time_dep = true;
                return clone(t->second);
            }
            auto d = doubles.find(temp);
            if (d != doubles.end()) {
                node->val = d->second;
                return node;
            }
            err = "No value " + temp + " found";
            return nullptr;
        }
        if (!ign.empty()) {
            int count = 0;
            for (int i = 0; i <= mop; ++i) {
                for (size_t j = 0; j < ign.size(); j += 2)
                    if (ign[j] == count) count += ign[j + 1] - ign[j] + 1;
                count++;
            }
            mop = count - 1;
        }
        if (mop < 0 || mop >= (int)s.size()) {
            err = "cannot split '" + s + "'";
            return nullptr;
        }
        node->op = operator_num(s[mop]);
        node->has_op = true;
        node->l = parse(s.substr(0, mop));
        node->r = parse(s.substr(mop + 1));
        return err.empty() ? node : nullptr;
    }
};

// tree_to_array: pre-order, right child only for op numbers below 6
void flatten(const std::shared_ptr<TNode>& n, std::vector<AstNode>& out) {
    const int idx = (int)out.size();
    AstNode a;
    a.val = n->val;
    a.is_dynamic = n->dyn ? 1 : 0;
    a.var = n->var;
    a.op_num = n->op;
    out.push_back(a);
    if (!n->has_op) return;
    out[idx].left = (int)out.size();
    flatten(n->l, out);
    if (n->op < 6) {
        out[idx].right = (int)out.size();
        flatten(n->r, out);
    }
}

// evaluate_eqn_gpu's walk as a postfix program
void lower(const std::vector<AstNode>& nodes, int k, std::vector<AstInstr>& prog, int sp,
           int& max_sp) {
    const AstNode& n = nodes[k];
    auto push = [&](AstInstr in) {
        prog.push_back(in);
        if (sp + 1 > max_sp) max_sp = sp + 1;
    };
    if (n.right < 0 && n.left < 0) {
        if (n.is_dynamic) {
            int code = n.var == 'x' ? AST_PUSH_X : n.var == 'y' ? AST_PUSH_Y
                     : n.var == 'z' ? AST_PUSH_Z : AST_PUSH_T;
            push({code, 0, 0.0});
        } else {
            push({AST_PUSH_CONST, 0, n.val});
        }
        return;
    }
    if (n.left > 0) lower(nodes, n.left, prog, sp, max_sp);
    else push({AST_PUSH_CONST, 0, 0.0});
    if (n.right > 0) lower(nodes, n.right, prog, sp + 1, max_sp);
    else {
        prog.push_back({AST_PUSH_CONST, 0, 0.0});
        if (sp + 2 > max_sp) max_sp = sp + 2;
    }
    prog.push_back({AST_OP, n.op_num, 0.0});
}

}  // namespace

static bool parse_into(const std::string& expr, const std::map<std::string, double>& doubles,
                       const std::map<std::string, std::shared_ptr<TNode>>& trees,
                       std::shared_ptr<TNode>& tree, AstExpr& out, std::string& err) {
    Parser p{doubles, trees};
    tree = p.parse(expr);
    if (!tree || !p.err.empty()) {
        err = p.err.empty() ? "parse failed" : p.err;
        return false;
    }
    out = AstExpr();
    out.time_dependent = p.time_dep;
    flatten(tree, out.nodes);
    int max_sp = 0;
    lower(out.nodes, 0, out.program, 0, max_sp);
    out.max_stack = max_sp;
    if (max_sp > kAstMaxStack || (int)out.program.size() > kAstMaxProgram) {
        err = "expression too large for the device evaluator";
        return false;
    }
    return true;
}

bool ast_parse(const std::string& expr, const std::map<std::string, double>& doubles,
               AstExpr& out, std::string& err) {
    std::map<std::string, std::shared_ptr<TNode>> none;
    std::shared_ptr<TNode> tree;
    return parse_into(expr, doubles, none, tree, out, err);
}

bool ast_parse_file(const std::string& text, const std::map<std::string, double>& doubles,
                    std::map<std::string, AstExpr>& out, std::vector<std::string>& order,
                    std::string& err) {
    std::map<std::string, std::shared_ptr<TNode>> trees;
    std::string val, eqn;
    auto allocate = [&](const std::string& name, const std::string& e) -> bool {
        std::shared_ptr<TNode> tree;
        AstExpr ex;
        if (!parse_into(e, doubles, trees, tree, ex, err)) {
            err = name + ": " + err;
            return false;
        }
        trees[name] = tree;
        out[name] = ex;
        bool seen = false;
        for (auto& o : order) seen |= (o == name);
        if (!seen) order.push_back(name);
        return true;
    };
    size_t pos = 0;
    while (pos <= text.size()) {
        size_t nl = text.find('\n', pos);
        std::string line = text.substr(pos, nl == std::string::npos ? std::string::npos : nl - pos);
        pos = (nl == std::string::npos) ? text.size() + 1 : nl + 1;
        std::string l;
        for (char ch : line)
            if (!std::isspace((unsigned char)ch)) l.push_back(ch);
        const size_t it = l.find('=');
        if (it == std::string::npos) {
            eqn += l;
        } else {
            if (!val.empty()) {
                if (val == "V") eqn += "+0.5*mass*(Ax*Ax+Ay*Ay+Az*Az)";
                if (!allocate(val, eqn)) return false;
                val.clear();
                eqn.clear();
            }
            val = l.substr(0, it);
            eqn = l.substr(it + 1);
        }
    }
    return allocate(val, eqn);
}

double ast_eval_host(const AstExpr& e, double x, double y, double z, double t) {
    return ast_eval(e.program.data(), (int)e.program.size(), x, y, z, t);
}

}  // namespace gpue
