/*
 * Helper.hpp -- drop-in for the reference's Helper.hpp (Helper.hpp:1-23,
 * Helper.cpp:3-9): DUMMY_VAL and utility::timer().
 *
 * The headers in this directory (Helper.hpp, EdgeList.hpp, CSCGraph.hpp,
 * CSRGraph.hpp, Graph.hpp, CountMat.hpp) give C++ callers of
 * dsc-nec/subgraph the reference's class names and method signatures on top
 * of the C ABI in ../sg_api.h, so that code written against the reference's
 * headers (its sc-main.cpp main, sc-main.cpp:1556-1805) compiles against them
 * and counts on the GPU.  Link with -lsubgraph_b200.  The reference reports no
 * errors; these classes throw sg_error (a std::runtime_error carrying the
 * library's status and message) when a library call fails.  Like the
 * reference's headers they bring namespace std into scope.
 */
#ifndef SUBGRAPH_B200_HELPER_HPP
#define SUBGRAPH_B200_HELPER_HPP

#include <sys/time.h>

#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "../sg_api.h"

using namespace std;

#ifndef DUMMY_VAL
#define DUMMY_VAL 93620
#endif

namespace utility {
inline double timer()
{
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return (double)tv.tv_sec + (double)tv.tv_usec * 1.0e-6;
}
}  // namespace utility

class sg_error : public std::runtime_error {
public:
    sg_error(sg_status code, const std::string &msg) : std::runtime_error(msg), code_(code) {}
    sg_status code() const { return code_; }

private:
    sg_status code_;
};

namespace sg_shim {
inline void check(sg_status st, const char *what)
{
    if (st != SG_OK) {
        const char *m = sg_last_error();
        throw sg_error(st, std::string(what) + ": " + (m ? m : ""));
    }
}

// a library-allocated array (sg_free) owned by a shim object
template <typename T> struct LibArray {
    T *p = nullptr;
    LibArray() = default;
    LibArray(const LibArray &) = delete;
    LibArray &operator=(const LibArray &) = delete;
    ~LibArray() { reset(nullptr); }
    void reset(T *q)
    {
        if (p) sg_free(p);
        p = q;
    }
};

// the device the shim's graphs are uploaded to: $SG_DEVICE, else 0
inline int32_t device()
{
    const char *e = std::getenv("SG_DEVICE");
    return e ? (int32_t)std::atoi(e) : 0;
}

// Host arrays of a CSC or CSR adjacency (offsets[V+1], neighbours in
// summation order, degrees) and its device copy, made on first use.
class Adjacency {
public:
    Adjacency() = default;
    Adjacency(const Adjacency &) = delete;
    Adjacency &operator=(const Adjacency &) = delete;
    ~Adjacency() { drop_device(); }

    int32_t V = -1, numEdges = -1;
    LibArray<int32_t> off, nbr, deg;

    void set(int32_t v, int32_t ne, int32_t *o, int32_t *n, int32_t *d)
    {
        drop_device();
        V = v;
        numEdges = ne;
        off.reset(o);
        nbr.reset(n);
        deg.reset(d);
    }
    int32_t nnz() const { return off.p ? off.p[V] : 0; }

    sg_graph device_graph()
    {
        if (!g_) {
            if (!off.p) throw sg_error(SG_ERR_INVALID, "graph used before it was created or loaded");
            check(sg_graph_create(off.p, nbr.p, V, nnz(), device(), &g_), "device graph");
        }
        return g_;
    }

    // graph.data bytes (CSCGraph.hpp:427-436 / CSRGraph.cpp:236-244)
    std::string encode() const
    {
        void *buf = nullptr;
        int64_t n = 0;
        check(sg_graph_data_encode(V, numEdges, off.p, nbr.p, deg.p, &buf, &n), "serialize");
        std::string out((const char *)buf, (size_t)n);
        sg_free(buf);
        return out;
    }
    void decode(const std::string &bytes)
    {
        int32_t v = 0, ne = 0, *o = nullptr, *n = nullptr, *d = nullptr;
        check(sg_graph_data_decode(bytes.data(), (int64_t)bytes.size(), &v, &ne, &o, &n, &d), "deserialize");
        set(v, ne, o, n, d);
    }

private:
    void drop_device()
    {
        if (g_) sg_graph_destroy(g_);
        g_ = nullptr;
    }
    sg_graph g_ = nullptr;
};

// the whole rest of a file descriptor (the reference's deserialize(int fd) reads it)
std::string read_fd(int fd);
}  // namespace sg_shim

#include <unistd.h>

inline std::string sg_shim::read_fd(int fd)
{
    std::string out;
    char buf[1 << 16];
    for (;;) {
        const ssize_t r = ::read(fd, buf, sizeof buf);
        if (r < 0) throw sg_error(SG_ERR_IO, "deserialize: read failed");
        if (r == 0) break;
        out.append(buf, (size_t)r);
    }
    return out;
}

#endif
