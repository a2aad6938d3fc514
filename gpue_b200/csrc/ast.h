// ast.h -- GPUE's equation strings: parser (host) and bytecode (device).
//
// GPUE reads "name = expr" lines from a parameter file (parse_param_file,
// src/dynamic.cu:187-222), parses each expression into a tree (parse_eqn,
// src/dynamic.cu:227-470), flattens it in pre-order (tree_to_array,
// src/dynamic.cu:472-507) and walks the flat array recursively on the device
// for every grid point (evaluate_eqn_gpu, src/dynamic.cu:527-603).  Here the
// same flat array is produced (so it can be compared node for node) and then
// lowered to a postfix program that a device stack machine runs per point;
// the arithmetic is the same operation sequence as the tree walk.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace gpue {

// Flat node, GPUE's EqnNode_gpu layout (include/ds.h:71-80).
struct AstNode {
    double val = 0.0;
    int32_t is_dynamic = 0;
    int32_t var = '0';
    int32_t left = -1, right = -1;
    int32_t op_num = 0;
};

// One postfix instruction.
enum AstOpcode : int32_t {
    AST_PUSH_CONST = 0,
    AST_PUSH_X = 1,
    AST_PUSH_Y = 2,
    AST_PUSH_Z = 3,
    AST_PUSH_T = 4,
    AST_OP = 5,  // applies op_num to the two topmost values (a = below, b = top)
};

struct AstInstr {
    int32_t code;
    int32_t op_num;
    double val;
};

constexpr int kAstMaxStack = 32;
constexpr int kAstMaxProgram = 512;

struct AstExpr {
    std::vector<AstNode> nodes;     // pre-order, GPUE layout
    std::vector<AstInstr> program;  // postfix
    int max_stack = 0;
    bool time_dependent = false;    // uses t or an earlier expression (GPUE's "_time")
};

// Parse one expression (whitespace already removed, as parse_param_file
// does).  doubles: the Grid doubles the expression may name.  Returns false
// with a message on failure (GPUE prints and exits instead).
bool ast_parse(const std::string& expr, const std::map<std::string, double>& doubles,
               AstExpr& out, std::string& err);

// parse_param_file on the text of a parameter file: V gets
// "+0.5*mass*(Ax*Ax+Ay*Ay+Az*Az)" appended unless it is the last entry.
bool ast_parse_file(const std::string& text, const std::map<std::string, double>& doubles,
                    std::map<std::string, AstExpr>& out, std::vector<std::string>& order,
                    std::string& err);

// Host evaluation of the postfix program (used by tests and checks).
double ast_eval_host(const AstExpr& e, double x, double y, double z, double t);

}  // namespace gpue
