// Test infrastructure (oracle): a minimal boost::dynamic_bitset<> stand-in that
// covers exactly the members the reference's CPU path touches: resize, reset,
// set, operator[] (read and write), &=, ==, count, find_first, find_next, npos,
// is_subset_of, size, the public block vector m_bits (the reference defines
// BOOST_DYNAMIC_BITSET_DONT_USE_FRIENDS and hashes m_bits directly), and
// operator<< for its debug printers.  Self-written; NOT Boost source.
//
// Invariant: bits at positions >= size() inside the last block are always zero,
// so block-wise equality and hashing agree with bit-wise equality.
#ifndef ORACLE_BOOST_SHIM_DYNAMIC_BITSET_HPP
#define ORACLE_BOOST_SHIM_DYNAMIC_BITSET_HPP

#include <cassert>
#include <climits>
#include <cstring>
#include <algorithm>
#include <cstddef>
#include <limits>
#include <ostream>
#include <vector>

#include "functional/hash.hpp"

namespace boost {

template <class Block = unsigned long> class dynamic_bitset {
  public:
    typedef Block block_type;
    typedef std::size_t size_type;
    static const size_type bits_per_block = std::numeric_limits<Block>::digits;
    static const size_type npos = static_cast<size_type>(-1);

    class reference {
      public:
        reference(block_type &b, block_type mask) : blk(b), msk(mask) {}
        operator bool() const { return (blk & msk) != 0; }
        reference &operator=(bool v) {
            if (v) {
                blk |= msk;
            } else {
                blk &= ~msk;
            }
            return *this;
        }
        reference &operator=(const reference &o) { return *this = static_cast<bool>(o); }

      private:
        block_type &blk;
        block_type msk;
    };

    // Public on purpose: the reference hashes the block vector directly.
    std::vector<block_type> m_bits;
    size_type m_num_bits;

    dynamic_bitset() : m_num_bits(0) {}
    explicit dynamic_bitset(size_type n, bool value = false) : m_num_bits(0) { resize(n, value); }

    size_type size() const { return m_num_bits; }

    void resize(size_type n, bool value = false) {
        const size_type old_bits = m_num_bits;
        m_bits.resize(blocks_for(n), block_type(0));
        m_num_bits = n;
        if (value) {
            for (size_type i = old_bits; i < n; ++i) {
                m_bits[i / bits_per_block] |= bit_mask(i);
            }
        }
        clear_tail();
    }

    dynamic_bitset &reset() {
        std::fill(m_bits.begin(), m_bits.end(), block_type(0));
        return *this;
    }

    dynamic_bitset &set(size_type pos, bool value = true) {
        assert(pos < m_num_bits);
        if (value) {
            m_bits[pos / bits_per_block] |= bit_mask(pos);
        } else {
            m_bits[pos / bits_per_block] &= ~bit_mask(pos);
        }
        return *this;
    }

    bool test(size_type pos) const {
        assert(pos < m_num_bits);
        return (m_bits[pos / bits_per_block] & bit_mask(pos)) != 0;
    }
    bool operator[](size_type pos) const { return test(pos); }
    reference operator[](size_type pos) {
        assert(pos < m_num_bits);
        return reference(m_bits[pos / bits_per_block], bit_mask(pos));
    }

    dynamic_bitset &operator&=(const dynamic_bitset &o) {
        assert(o.m_num_bits == m_num_bits);
        for (size_type i = 0; i < m_bits.size(); ++i) {
            m_bits[i] &= o.m_bits[i];
        }
        return *this;
    }

    size_type count() const {
        size_type c = 0;
        for (size_type i = 0; i < m_bits.size(); ++i) {
            c += static_cast<size_type>(__builtin_popcountl(static_cast<unsigned long>(m_bits[i])));
        }
        return c;
    }

    size_type find_first() const { return find_from(0); }
    size_type find_next(size_type pos) const {
        if (pos == npos || pos + 1 >= m_num_bits) {
            return npos;
        }
        return find_from(pos + 1);
    }

    bool is_subset_of(const dynamic_bitset &o) const {
        assert(o.m_num_bits == m_num_bits);
        for (size_type i = 0; i < m_bits.size(); ++i) {
            if ((m_bits[i] & ~o.m_bits[i]) != 0) {
                return false;
            }
        }
        return true;
    }

    bool operator==(const dynamic_bitset &o) const {
        return m_num_bits == o.m_num_bits && m_bits == o.m_bits;
    }
    bool operator!=(const dynamic_bitset &o) const { return !(*this == o); }

  private:
    static size_type blocks_for(size_type n) { return (n + bits_per_block - 1) / bits_per_block; }
    static block_type bit_mask(size_type pos) { return block_type(1) << (pos % bits_per_block); }

    void clear_tail() {
        const size_type extra = m_num_bits % bits_per_block;
        if (extra != 0 && !m_bits.empty()) {
            m_bits.back() &= (block_type(1) << extra) - 1;
        }
    }

    size_type find_from(size_type pos) const {
        if (pos >= m_num_bits) {
            return npos;
        }
        size_type blk = pos / bits_per_block;
        block_type word = m_bits[blk] & (~block_type(0) << (pos % bits_per_block));
        while (true) {
            if (word != 0) {
                return blk * bits_per_block +
                       static_cast<size_type>(__builtin_ctzl(static_cast<unsigned long>(word)));
            }
            ++blk;
            if (blk >= m_bits.size()) {
                return npos;
            }
            word = m_bits[blk];
        }
    }
};

template <class B> const typename dynamic_bitset<B>::size_type dynamic_bitset<B>::bits_per_block;
template <class B> const typename dynamic_bitset<B>::size_type dynamic_bitset<B>::npos;

// Prints most-significant bit first, like Boost's stream operator.
template <class B> std::ostream &operator<<(std::ostream &os, const dynamic_bitset<B> &b) {
    for (std::size_t i = b.size(); i-- > 0;) {
        os << (b.test(i) ? '1' : '0');
    }
    return os;
}

} // namespace boost

#endif
