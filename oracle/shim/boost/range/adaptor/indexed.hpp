/*
 * Test infrastructure (oracle): a minimal stand-in for boost::adaptors::indexed, which the
 * LPM-CPP reference uses as `range | indexed(0)` inside `#pragma omp parallel for` loops
 * (include/stiffness.h:203,207,297,301,390).  Boost is not installed on this machine.
 *
 * The element exposes index() and value(); the iterator is random-access so that GCC's
 * OpenMP range-for lowering (which needs operator-, operator+= and operator<) accepts it.
 */
#pragma once
#ifndef LPM_ORACLE_BOOST_INDEXED_SHIM
#define LPM_ORACLE_BOOST_INDEXED_SHIM

#include <cstddef>
#include <iterator>

namespace boost
{
namespace adaptors
{

template <class It>
struct index_value
{
    std::ptrdiff_t idx;
    It it;
    std::ptrdiff_t index() const { return idx; }
    decltype(*std::declval<It>()) value() const { return *it; }
};

template <class It>
class indexed_iterator
{
public:
    using iterator_category = std::random_access_iterator_tag;
    using value_type = index_value<It>;
    using difference_type = std::ptrdiff_t;
    using pointer = void;
    using reference = value_type;

    indexed_iterator() = default;
    indexed_iterator(It it, std::ptrdiff_t idx) : it_(it), idx_(idx) {}

    value_type operator*() const { return value_type{idx_, it_}; }
    value_type operator[](difference_type n) const { return value_type{idx_ + n, it_ + n}; }

    indexed_iterator &operator++() { ++it_; ++idx_; return *this; }
    indexed_iterator operator++(int) { indexed_iterator t = *this; ++*this; return t; }
    indexed_iterator &operator--() { --it_; --idx_; return *this; }
    indexed_iterator operator--(int) { indexed_iterator t = *this; --*this; return t; }
    indexed_iterator &operator+=(difference_type n) { it_ += n; idx_ += n; return *this; }
    indexed_iterator &operator-=(difference_type n) { it_ -= n; idx_ -= n; return *this; }
    friend indexed_iterator operator+(indexed_iterator a, difference_type n) { a += n; return a; }
    friend indexed_iterator operator+(difference_type n, indexed_iterator a) { a += n; return a; }
    friend indexed_iterator operator-(indexed_iterator a, difference_type n) { a -= n; return a; }
    friend difference_type operator-(const indexed_iterator &a, const indexed_iterator &b) { return a.it_ - b.it_; }
    friend bool operator==(const indexed_iterator &a, const indexed_iterator &b) { return a.it_ == b.it_; }
    friend bool operator!=(const indexed_iterator &a, const indexed_iterator &b) { return a.it_ != b.it_; }
    friend bool operator<(const indexed_iterator &a, const indexed_iterator &b) { return a.it_ < b.it_; }
    friend bool operator>(const indexed_iterator &a, const indexed_iterator &b) { return a.it_ > b.it_; }
    friend bool operator<=(const indexed_iterator &a, const indexed_iterator &b) { return a.it_ <= b.it_; }
    friend bool operator>=(const indexed_iterator &a, const indexed_iterator &b) { return a.it_ >= b.it_; }

private:
    It it_{};
    std::ptrdiff_t idx_{0};
};

template <class It>
struct indexed_range
{
    indexed_iterator<It> b, e;
    indexed_iterator<It> begin() const { return b; }
    indexed_iterator<It> end() const { return e; }
};

struct indexed
{
    std::ptrdiff_t base;
    explicit indexed(std::ptrdiff_t p_base = 0) : base(p_base) {}
};

template <class R>
auto operator|(R &r, const indexed &ix) -> indexed_range<decltype(r.begin())>
{
    using It = decltype(r.begin());
    std::ptrdiff_t n = r.end() - r.begin();
    return indexed_range<It>{indexed_iterator<It>(r.begin(), ix.base), indexed_iterator<It>(r.end(), ix.base + n)};
}

} // namespace adaptors
} // namespace boost

#endif
