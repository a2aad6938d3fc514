// grid.h -- the parameter store the host layer passes around, after GPUE's
// Grid class (include/ds.h:86-196): typed maps of named ints, doubles, bools
// and strings, the field-function names (-A, -v), the coordinate axes and
// the host copy of the wavefunction.  A missing key throws with its name
// (GPUE asserts, src/ds.cu:186-265).
#pragma once

#include <complex>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/gpue_b200.h"

namespace gpue_host {

class Grid {
   public:
    void store(const std::string& k, int v) { ints_[k] = v; }
    void store(const std::string& k, double v) { doubles_[k] = v; }
    void store(const std::string& k, bool v) { bools_[k] = v; }
    void store(const std::string& k, const std::string& v) { strings_[k] = v; }
    void store(const std::string& k, const char* v) { strings_[k] = v; }

    int ival(const std::string& k) const { return get(ints_, k, "int"); }
    double dval(const std::string& k) const { return get(doubles_, k, "double"); }
    bool bval(const std::string& k) const { return get(bools_, k, "bool"); }
    std::string sval(const std::string& k) const { return get(strings_, k, "string"); }
    bool has(const std::string& k) const {
        return ints_.count(k) || doubles_.count(k) || bools_.count(k) || strings_.count(k);
    }

    // Params.dat: "[Params]" then one key=value line per stored scalar, as
    // GPUE's Grid::write (src/ds.cu:269-288)
    void write(const std::string& file) const;

    std::string Afn = "rotation";  // gauge field (-A)
    std::string Kfn = "rotation_K";
    std::string Vfn = "2d";        // potential (-v)
    std::string Wfcfn = "2d";

    std::vector<double> x, y, z;                // positions (generate_p_space)
    std::vector<std::complex<double>> wfc;      // host wavefunction, x fastest

    // The library context the evolve() shim keeps for this Grid.
    gpue_ctx* ctx() const { return ctx_ ? ctx_->c : nullptr; }
    void set_ctx(gpue_ctx* c) { ctx_ = std::make_shared<Ctx>(c); }

   private:
    struct Ctx {
        explicit Ctx(gpue_ctx* p) : c(p) {}
        ~Ctx() {
            if (c) gpue_ctx_destroy(c);
        }
        Ctx(const Ctx&) = delete;
        Ctx& operator=(const Ctx&) = delete;
        gpue_ctx* c;
    };

    template <typename M>
    static typename M::mapped_type get(const M& m, const std::string& k, const char* what) {
        auto it = m.find(k);
        if (it == m.end()) throw std::out_of_range(std::string("Grid: no ") + what + " '" + k + "'");
        return it->second;
    }

    std::map<std::string, int> ints_;
    std::map<std::string, double> doubles_;
    std::map<std::string, bool> bools_;
    std::map<std::string, std::string> strings_;
    std::shared_ptr<Ctx> ctx_;
};

}  // namespace gpue_host
