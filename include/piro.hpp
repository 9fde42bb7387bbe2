// piro.hpp -- PIRO's C++ operator spelling over the C ABI of piro.h.
//
// A solve.cpp written against PIRO keeps its equations unchanged:
//
//     Piro::Case run(assets_dir, "HeatEq.ini");
//     Piro::process solver(run);
//     float time = 0.0f;
//     while (time < run.info().totaltime) {
//         Piro::scalarMatrix UEqn(solver.ddt_r("T") = solver.laplacian("T", "Alpha"));
//         UEqn.Solve(time);
//         time += run.info().timestep;
//     }
//
// (src/solve.cpp:11-48).  Errors become Piro::Error exceptions carrying the
// status code and piro_last_error(); nothing is thrown across the C ABI itself.
#pragma once

#include <stdexcept>
#include <string>

#include "piro.h"

namespace Piro {

struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string &where)
        : std::runtime_error(where + ": " + piro_status_string(s) + ": " + piro_last_error()), status(s)
    {
    }
};

inline void check(int s, const char *where)
{
    if (s != PIRO_OK) throw Error(s, where);
}

class Case {
  public:
    Case(const std::string &assets_dir, const std::string &case_name)
    {
        check(piro_open(assets_dir.c_str(), case_name.c_str(), &ctx_), "piro_open");
    }
    ~Case() { piro_close(ctx_); }
    Case(const Case &) = delete;
    Case &operator=(const Case &) = delete;
    piro_ctx *get() const { return ctx_; }
    piro_case_info info() const
    {
        piro_case_info i;
        check(piro_ctx_query(ctx_, &i), "piro_ctx_query");
        return i;
    }

  private:
    piro_ctx *ctx_ = nullptr;
};

class Operator {
  public:
    Operator(piro_ctx *c, piro_op o) : ctx(c), op(o) {}
    piro_ctx *ctx;
    piro_op op;
};

// CLBuffer (operatoroverload.hpp:9-17): a field; operator= runs the time scheme.
class CLBuffer {
  public:
    CLBuffer(piro_ctx *c, piro_buf b) : ctx(c), buf(b) {}
    CLBuffer operator=(const Operator &rhs)
    {
        piro_buf out;
        check(piro_assign(ctx, buf, rhs.op, &out), "piro_assign");
        return CLBuffer(ctx, out);
    }
    piro_ctx *ctx;
    piro_buf buf;
};

// operator& (operatoroverload.cpp:102-123): vector & gradient.
inline Operator operator&(const CLBuffer &v, const Operator &grad)
{
    piro_op out;
    check(piro_dot(v.ctx, v.buf, grad.op, &out), "piro_dot");
    return Operator(v.ctx, out);
}

class process {
  public:
    explicit process(Case &c) : ctx_(c.get()) {}
    CLBuffer ddt_r(const std::string &var)
    {
        piro_buf b;
        check(piro_ddt_r(ctx_, var.c_str(), &b), "piro_ddt_r");
        return CLBuffer(ctx_, b);
    }
    CLBuffer vector(const std::string &var)
    {
        piro_buf b;
        check(piro_vector(ctx_, var.c_str(), &b), "piro_vector");
        return CLBuffer(ctx_, b);
    }
    Operator laplacian(const std::string &var, const std::string &coeff)
    {
        piro_op o;
        check(piro_laplacian(ctx_, var.c_str(), coeff.c_str(), &o), "piro_laplacian");
        return Operator(ctx_, o);
    }
    Operator gradient(const std::string &var)
    {
        piro_op o;
        check(piro_gradient(ctx_, var.c_str(), &o), "piro_gradient");
        return Operator(ctx_, o);
    }

  private:
    piro_ctx *ctx_;
};

class scalarMatrix {
  public:
    explicit scalarMatrix(const CLBuffer &eqn) : eqn_(eqn) {}
    void Solve(float time) { check(piro_step_solve(eqn_.ctx, eqn_.buf, time), "piro_step_solve"); }

  private:
    CLBuffer eqn_;
};

}  // namespace Piro
