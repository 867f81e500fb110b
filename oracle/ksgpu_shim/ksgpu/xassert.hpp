// Minimal stand-in for ksgpu's assertion macros (TEST INFRASTRUCTURE ONLY; see Array.hpp): a failed
// check throws std::runtime_error naming the expression, file and line.
#pragma once

#include <sstream>
#include <stdexcept>

#define xassert(cond) \
    do { \
        if (!(cond)) { \
            std::stringstream ss_; \
            ss_ << "assertion failed: " << #cond << " (" << __FILE__ << ":" << __LINE__ << ")"; \
            throw std::runtime_error(ss_.str()); \
        } \
    } while (0)

#define xassert_cmp_(a, b, op) \
    do { \
        const auto a_ = (a); \
        const auto b_ = (b); \
        if (!(a_ op b_)) { \
            std::stringstream ss_; \
            ss_ << "assertion failed: " << #a << " " #op " " << #b << " (" << a_ << " vs " << b_ << ", " \
                << __FILE__ << ":" << __LINE__ << ")"; \
            throw std::runtime_error(ss_.str()); \
        } \
    } while (0)

#define xassert_eq(a, b) xassert_cmp_(a, b, ==)
#define xassert_ne(a, b) xassert_cmp_(a, b, !=)
#define xassert_le(a, b) xassert_cmp_(a, b, <=)
#define xassert_lt(a, b) xassert_cmp_(a, b, <)
#define xassert_ge(a, b) xassert_cmp_(a, b, >=)
#define xassert_gt(a, b) xassert_cmp_(a, b, >)
