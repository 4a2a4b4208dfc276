// Minimal stand-in for pyre's grid and memory packages (test infrastructure: it lets the
// reference's CPU correlator, lib/libampcor/correlators/Sequential.cc with Sequential.icc and
// SumArea.icc, and its SLC raster, lib/libampcor/dom/SLC.icc, compile unmodified).
//
// What the reference relies on, and how it is provided here:
//
// * index_t<std::array<size_t, D>>: a D-tuple with element-wise + and -, fill(v), begin()/end()
//   over its elements and [] access; braces {a, b} build one.
// * layout_t<index_t>: a shape, a low corner (zero) and a packing order, the list of axes from
//   the fastest varying to the slowest; the default packing is row-major ({D-1, ..., 0}), the
//   order pyre's SLC states explicitly ({1, 0}, SLC.icc:122-126).  offset(index) is
//   sum_k (index[p_k] - low[p_k]) * prod_{j<k} shape[p_j].
// * slice_t: a [low, high) box of a layout with its packing.  Iterating a layout or a slice
//   follows pyre's iterator: start at low; to advance, walk the axes in packing order,
//   increment the index on that axis and stop if it is still below high on that axis, else
//   reset it to low and carry into the next axis; when every axis has carried, the iterator
//   becomes high, which is the end.  A box that is flat on a slow axis (high == low there) is
//   therefore walked along its fast axes once: SumArea's constructor (SumArea.icc:158-176) fills
//   the first row and the first column of a table through slices from low + h to
//   {low[0], high[1]} and from low + v to {high[0], low[1]}, which is what this gives.
// * grid_t<cell, layout, storage>: a layout over storage; [] by offset or by index; view() and
//   view(slice) iterate cells in the layout's or slice's order; a grid can be built from a layout
//   alone (heap storage, converting constructor: Sequential.cc:48 and Correlator.icc:40 build
//   their summed-area table from `tgt.layout()`, that is from a new grid of the window's layout),
//   from a layout and a cell pointer (view storage) or, for directgrid_t, from a file name and a
//   layout (a read-only memory map of a raw raster file).
// * heap_t: cells from the heap.  pyre allocates them with new[]; whether that storage starts out
//   zero is not something the reference's code states.  Here it is value-initialised (zero), so
//   that a table built over a new grid is the same on every run.
#ifndef AMPCOR_REF_SHIM_PYRE_GRID_H
#define AMPCOR_REF_SHIM_PYRE_GRID_H

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <array>
#include <complex>
#include <cstddef>
#include <iterator>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>

namespace pyre {

namespace memory {

using uri_t = std::string;

// cells owned on the heap (value-initialised)
template <typename cellT>
class heap_t {
public:
    using cell_type = cellT;
    explicit heap_t(std::size_t cells) : _cells(new cell_type[cells]()) {}
    cell_type* data() const { return _cells.get(); }

private:
    std::shared_ptr<cell_type[]> _cells;
};

// cells owned elsewhere
template <typename cellT>
class view_t {
public:
    using cell_type = cellT;
    view_t(cell_type* cells) : _cells(cells) {}
    cell_type* data() const { return _cells; }

private:
    cell_type* _cells;
};

template <typename cellT>
class constview_t {
public:
    using cell_type = const cellT;
    constview_t(const cellT* cells) : _cells(cells) {}
    const cellT* data() const { return _cells; }

private:
    const cellT* _cells;
};

// a read-only memory map of a raw file of cells
template <typename cellT>
class constdirect_t {
public:
    using cell_type = const cellT;
    constdirect_t(const uri_t& name, std::size_t cells)
    {
        const std::size_t bytes = cells * sizeof(cellT);
        const int fd = ::open(name.c_str(), O_RDONLY);
        if (fd < 0) throw std::runtime_error("cannot open " + name);
        struct stat st {};
        if (::fstat(fd, &st) != 0 || (std::size_t)st.st_size < bytes) {
            ::close(fd);
            throw std::runtime_error(name + " is smaller than its shape");
        }
        void* p = bytes ? ::mmap(nullptr, bytes, PROT_READ, MAP_SHARED, fd, 0) : nullptr;
        ::close(fd);
        if (p == MAP_FAILED) throw std::runtime_error("cannot map " + name);
        _map = std::shared_ptr<void>(p, [bytes](void* q) {
            if (q) ::munmap(q, bytes);
        });
    }
    const cellT* data() const { return static_cast<const cellT*>(_map.get()); }

private:
    std::shared_ptr<void> _map;
};

}  // namespace memory

namespace grid {

template <typename repT>
class index_t {
public:
    using rep_type = repT;
    using value_type = typename repT::value_type;
    using size_type = std::size_t;

    static constexpr size_type dim() { return std::tuple_size<repT>::value; }

    index_t() : _rep{} {}
    template <typename... T,
              typename = std::enable_if_t<sizeof...(T) == std::tuple_size<repT>::value &&
                                          (std::is_arithmetic_v<T> && ...)>>
    index_t(T... v) : _rep{{static_cast<value_type>(v)...}}
    {
    }

    static index_t fill(value_type v)
    {
        index_t r;
        r._rep.fill(v);
        return r;
    }

    value_type& operator[](size_type i) { return _rep[i]; }
    const value_type& operator[](size_type i) const { return _rep[i]; }
    auto begin() const { return _rep.begin(); }
    auto end() const { return _rep.end(); }
    auto begin() { return _rep.begin(); }
    auto end() { return _rep.end(); }

    friend index_t operator+(const index_t& a, const index_t& b)
    {
        index_t r;
        for (size_type k = 0; k < dim(); ++k) r._rep[k] = a._rep[k] + b._rep[k];
        return r;
    }
    friend index_t operator-(const index_t& a, const index_t& b)
    {
        index_t r;
        for (size_type k = 0; k < dim(); ++k) r._rep[k] = a._rep[k] - b._rep[k];
        return r;
    }
    friend bool operator==(const index_t& a, const index_t& b) { return a._rep == b._rep; }
    friend bool operator!=(const index_t& a, const index_t& b) { return !(a == b); }
    friend std::ostream& operator<<(std::ostream& os, const index_t& x)
    {
        for (size_type k = 0; k < dim(); ++k) os << (k ? ", " : "") << x._rep[k];
        return os;
    }

private:
    repT _rep;
};

// pyre's iterator over a box [low, high) in packing order (see the header comment)
template <typename indexT>
class box_iterator_t {
public:
    using iterator_category = std::forward_iterator_tag;
    using value_type = indexT;
    using difference_type = std::ptrdiff_t;
    using pointer = const indexT*;
    using reference = const indexT&;

    box_iterator_t(indexT current, indexT low, indexT high, indexT packing)
        : _current(current), _low(low), _high(high), _packing(packing)
    {
    }
    reference operator*() const { return _current; }
    pointer operator->() const { return &_current; }
    box_iterator_t& operator++()
    {
        for (auto axis : _packing) {
            if (++_current[axis] < _high[axis]) return *this;
            _current[axis] = _low[axis];
        }
        _current = _high;
        return *this;
    }
    box_iterator_t operator++(int)
    {
        box_iterator_t r = *this;
        ++*this;
        return r;
    }
    friend bool operator==(const box_iterator_t& a, const box_iterator_t& b) { return a._current == b._current; }
    friend bool operator!=(const box_iterator_t& a, const box_iterator_t& b) { return !(a == b); }

private:
    indexT _current, _low, _high, _packing;
};

template <typename indexT>
class slice_t {
public:
    using index_type = indexT;
    using shape_type = indexT;
    using packing_type = indexT;
    using iterator = box_iterator_t<indexT>;

    slice_t(index_type low, index_type high, packing_type packing)
        : _low(low), _high(high), _packing(packing)
    {
    }
    const index_type& low() const { return _low; }
    const index_type& high() const { return _high; }
    shape_type shape() const { return _high - _low; }
    const packing_type& packing() const { return _packing; }
    iterator begin() const { return iterator(_low, _low, _high, _packing); }
    iterator end() const { return iterator(_high, _low, _high, _packing); }

private:
    index_type _low, _high;
    packing_type _packing;
};

template <typename indexT>
class layout_t {
public:
    using index_type = indexT;
    using shape_type = indexT;
    using packing_type = indexT;
    using slice_type = slice_t<indexT>;
    using size_type = std::size_t;
    using iterator = box_iterator_t<indexT>;

    static constexpr size_type dim() { return indexT::dim(); }

    static packing_type rowMajor()
    {
        packing_type p;
        for (size_type k = 0; k < dim(); ++k) p[k] = dim() - 1 - k;
        return p;
    }

    layout_t(shape_type shape, packing_type packing = rowMajor())
        : _shape(shape), _low(), _packing(packing)
    {
        size_type stride = 1;
        for (auto axis : _packing) {
            _stride[axis] = stride;
            stride *= _shape[axis];
        }
    }

    const shape_type& shape() const { return _shape; }
    const packing_type& packing() const { return _packing; }
    index_type low() const { return _low; }
    index_type high() const { return _low + _shape; }
    size_type size() const
    {
        size_type n = 1;
        for (auto s : _shape) n *= s;
        return n;
    }
    // the strides are those of the packing order, computed once
    size_type offset(const index_type& index) const
    {
        size_type off = 0;
        for (size_type k = 0; k < dim(); ++k) off += (index[k] - _low[k]) * _stride[k];
        return off;
    }
    slice_type slice(const index_type& low, const index_type& high) const { return slice_type(low, high, _packing); }
    iterator begin() const { return iterator(_low, _low, high(), _packing); }
    iterator end() const { return iterator(high(), _low, high(), _packing); }

private:
    shape_type _shape;
    index_type _low;
    packing_type _packing;
    std::array<size_type, indexT::dim()> _stride{};
};

// the cells of a grid in the order of a box of its layout
template <typename gridT, typename refT>
class grid_view_t {
public:
    using slice_type = typename gridT::slice_type;
    using index_iterator = typename slice_type::iterator;

    class iterator {
    public:
        using iterator_category = std::forward_iterator_tag;
        using value_type = std::remove_cv_t<std::remove_reference_t<refT>>;
        using difference_type = std::ptrdiff_t;
        using pointer = std::remove_reference_t<refT>*;
        using reference = refT;

        iterator(const gridT* g, index_iterator it) : _g(g), _it(it) {}
        reference operator*() const { return const_cast<gridT*>(_g)->cell(*_it); }
        iterator& operator++()
        {
            ++_it;
            return *this;
        }
        iterator operator++(int)
        {
            iterator r = *this;
            ++_it;
            return r;
        }
        friend bool operator==(const iterator& a, const iterator& b) { return a._it == b._it; }
        friend bool operator!=(const iterator& a, const iterator& b) { return !(a == b); }

    private:
        const gridT* _g;
        index_iterator _it;
    };

    grid_view_t(const gridT* g, slice_type s) : _g(g), _slice(s) {}
    iterator begin() const { return iterator(_g, _slice.begin()); }
    iterator end() const { return iterator(_g, _slice.end()); }
    const slice_type& slice() const { return _slice; }
    const typename gridT::layout_type& layout() const { return _g->layout(); }

private:
    const gridT* _g;
    slice_type _slice;
};

template <typename cellT, typename layoutT, typename storageT>
class grid_t {
public:
    using cell_type = cellT;
    using layout_type = layoutT;
    using storage_type = storageT;
    using index_type = typename layoutT::index_type;
    using shape_type = typename layoutT::shape_type;
    using packing_type = typename layoutT::packing_type;
    using slice_type = typename layoutT::slice_type;
    using size_type = std::size_t;
    using cell_ref = std::conditional_t<std::is_const_v<typename storageT::cell_type>, const cellT&, cellT&>;
    using view_type = grid_view_t<grid_t, cell_ref>;
    using constview_type = grid_view_t<grid_t, const cellT&>;

    static constexpr size_type dim() { return layoutT::dim(); }

    // a grid of a layout on the heap (a converting constructor, as in pyre)
    template <typename S = storageT, typename = std::enable_if_t<std::is_same_v<S, memory::heap_t<cellT>>>>
    grid_t(layout_type layout) : _layout(layout), _storage(layout.size())
    {
    }
    // a grid of a layout over cells owned elsewhere
    template <typename P, typename S = storageT,
              typename = std::enable_if_t<!std::is_same_v<S, memory::heap_t<cellT>> &&
                                          std::is_constructible_v<S, P>>>
    grid_t(layout_type layout, P cells) : _layout(layout), _storage(cells)
    {
    }

    const layout_type& layout() const { return _layout; }
    auto data() const { return _storage.data(); }

    cell_ref operator[](size_type offset) const { return const_cast<cell_ref>(_storage.data()[offset]); }
    cell_ref operator[](const index_type& index) const { return cell(index); }
    cell_ref cell(const index_type& index) const
    {
        return const_cast<cell_ref>(_storage.data()[_layout.offset(index)]);
    }

    view_type view() const { return view_type(this, _layout.slice(_layout.low(), _layout.high())); }
    view_type view(const slice_type& slice) const { return view_type(this, slice); }
    constview_type constview(const slice_type& slice) const { return constview_type(this, slice); }

protected:
    grid_t(layout_type layout, storage_type storage) : _layout(layout), _storage(std::move(storage)) {}

private:
    layout_type _layout;
    storage_type _storage;
};

// a grid over a memory-mapped raw file: directgrid_t(uri, layout)
template <typename cellT, typename layoutT, typename storageT = memory::constdirect_t<cellT>>
class directgrid_t : public grid_t<cellT, layoutT, storageT> {
public:
    using base_type = grid_t<cellT, layoutT, storageT>;
    using typename base_type::layout_type;
    directgrid_t(const memory::uri_t& name, layout_type layout)
        : base_type(layout, storageT(name, layout.size()))
    {
    }
};

}  // namespace grid
}  // namespace pyre

#endif
