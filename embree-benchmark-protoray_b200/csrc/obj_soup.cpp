// OBJ -> triangle soup on host threads: the input stage of `protoray build`.
//
// Replaces ObjLoader (main/build/obj_loader.cpp), which reads the file with
// one fscanf/fgets pair per line on one thread.  Here the file is read whole,
// cut into chunks at line boundaries and parsed in three passes:
//   1. per chunk, in parallel: v / vn / vt values, face corners as written
//      (indices not yet resolved) and usemtl events, with the chunk-local
//      list sizes at each face;
//   2. serially over chunks: list bases and material ids, so that a face's
//      relative (negative) index and current material resolve exactly as in a
//      single pass over the file (obj_loader.cpp:194-226, 229-244);
//   3. per chunk, in parallel: fan triangulation, dropping triangles with two
//      equal position indices (:211-221), index validation against the final
//      list sizes (makeSoup, :253-324), and output at each chunk's triangle
//      offset (counted in a first sweep, written in a second).
// The result is identical to the reference loader's soup, triangle for
// triangle.  Differences only where the reference has undefined behaviour:
// a position index of 0 (it reads positionList[-1]) is rejected, and lines
// are not split at 256 KiB.
#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <unistd.h>

#include "../../include/prt_b200.h"
#include "soup_view.h"

namespace {

// Large host buffers (the file text, the soup) on 2 MiB-aligned memory with
// transparent huge pages requested: a 138 MB soup is then 69 page faults, not
// 34,000, and the threads that write it do not queue on the page-table lock.
struct HugeFree
{
    void operator()(void* p) const { std::free(p); }
};

void* huge_alloc(size_t bytes)
{
    const size_t align = size_t(2) << 20;
    const size_t n = (std::max<size_t>(bytes, 1) + align - 1) / align * align;
    void* p = std::aligned_alloc(align, n);
    if (p) madvise(p, n, MADV_HUGEPAGE);
    return p;
}

} // namespace

// A parsed OBJ: its vertex lists, each triangle's resolved corner indices and
// material id (the indexed form the GPU builder uploads), and the expanded
// 100-byte triangle records, made on the first prt_soup_triangles call.
struct prt_soup
{
    std::vector<float> v, vt, vn;
    std::unique_ptr<int, HugeFree> corners;   // 3 x cornerInts per triangle
    std::unique_ptr<int, HugeFree> mat;
    int cornerInts = 1;
    long long triCount = 0;
    std::vector<std::string> names;
    long long degenerate = 0;
    std::unique_ptr<prt_soup_triangle, HugeFree> tris;   // expanded on demand
};

namespace {

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f' || c == '\n'; }
// strtok delimiters of the face parser (obj_loader.cpp:163)
inline bool is_face_delim(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }

// Decimal -> float with the result of strtof, for the common case.  A
// decimal number w x 10^q with w < 2^53 and |q| <= 22 converts to the nearest
// double with one IEEE multiply or divide of exact operands (Clinger,
// "How to read floating point numbers accurately", PLDI 1990).  Rounding that
// double to float gives the nearest float unless the double lies exactly on a
// midpoint between two floats (every float midpoint is a double, so no other
// midpoint can separate the double from the exact value); that case, numbers
// outside the normal float range, more than 19 significant digits, hex,
// inf and nan return false and are left to strtof.  On success `next` is the
// first character after the number, as strtof's end pointer.
bool fast_decimal_float(const char* s, const char* end, float& out, const char*& next)
{
    static const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                      1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};
    const char* p = s;
    bool neg = false;
    if (p < end && (*p == '+' || *p == '-')) neg = *p++ == '-';
    if (p + 1 < end && p[0] == '0' && (p[1] == 'x' || p[1] == 'X')) return false;
    uint64_t w = 0;
    int digits = 0, q = 0;
    bool any = false;
    while (p < end && *p >= '0' && *p <= '9')
    {
        any = true;
        if (w != 0 || *p != '0')
        {
            if (++digits > 19) return false;
            w = w * 10 + (uint64_t)(*p - '0');
        }
        ++p;
    }
    if (p < end && *p == '.')
    {
        ++p;
        while (p < end && *p >= '0' && *p <= '9')
        {
            any = true;
            if (w != 0 || *p != '0')
            {
                if (++digits > 19) return false;
                w = w * 10 + (uint64_t)(*p - '0');
            }
            --q;
            ++p;
        }
    }
    if (!any) return false;
    if (p < end && (*p == 'e' || *p == 'E'))
    {
        const char* e = p + 1;
        bool eneg = false;
        if (e < end && (*e == '+' || *e == '-')) eneg = *e++ == '-';
        if (e < end && *e >= '0' && *e <= '9')
        {
            int x = 0;
            while (e < end && *e >= '0' && *e <= '9')
            {
                if (x < 100000) x = x * 10 + (*e - '0');
                ++e;
            }
            q += eneg ? -x : x;
            p = e;
        }
    }
    next = p;
    if (w == 0)
    {
        out = neg ? -0.0f : 0.0f;
        return true;
    }
    if (w > (1ULL << 53) || q < -22 || q > 22) return false;
    double d = (double)w;
    d = q >= 0 ? d * kPow10[q] : d / kPow10[-q];
    if (d > 3.4028234663852886e38 || d < 1.1754943508222875e-38) return false;   // overflow or subnormal
    uint64_t bits;
    std::memcpy(&bits, &d, 8);
    if ((bits & ((1ULL << 29) - 1)) == (1ULL << 28)) return false;   // exactly halfway between two floats
    out = neg ? -(float)d : (float)d;
    return true;
}

// sscanf "%f": skips white space, then converts as strtof.  `end` bounds the line.
bool scan_float(const char*& s, const char* end, float& out)
{
    while (s < end && is_ws(*s)) ++s;
    if (s >= end) return false;
    const char* next = nullptr;
    if (fast_decimal_float(s, end, out, next))
    {
        s = next;
        return true;
    }
    char* e = nullptr;
    out = std::strtof(s, &e);
    if (e == s || e > end) return false;
    s = e;
    return true;
}

// sscanf "%d" within [s, end): optional sign and decimal digits.
bool scan_int(const char*& s, const char* end, int& out)
{
    const char* p = s;
    while (p < end && (*p == '\v' || *p == '\f')) ++p;
    bool neg = false;
    if (p < end && (*p == '+' || *p == '-')) neg = *p++ == '-';
    if (p >= end || *p < '0' || *p > '9') return false;
    long long v = 0;
    while (p < end && *p >= '0' && *p <= '9')
        v = std::min(v * 10 + (*p++ - '0'), 1LL << 31);   // saturates: an out-of-range index
    out = neg ? (int)std::max(-v, -(1LL << 31)) : (int)std::min(v, 0x7fffffffLL);
    s = p;
    return true;
}

// One corner token, tried against the reference's four patterns in order
// (obj_loader.cpp:170-194): p/t/n, p//n, p/t, p.  Returns false if none match.
bool scan_corner(const char* s, const char* end, int& p, int& t, int& n)
{
    const char* q = s;
    int a, b, c;
    if (!scan_int(q, end, a)) return false;
    if (q >= end || *q != '/')
    {
        // a plain position index: every pattern stops after the first number
        p = a;
        t = 0;
        n = 0;
        return true;
    }
    // "%d/%d/%d"
    {
        const char* r = q + 1;
        if (scan_int(r, end, b) && r < end && *r == '/')
        {
            const char* u = r + 1;
            if (scan_int(u, end, c))
            {
                p = a;
                t = b;
                n = c;
                return true;
            }
        }
        // "%d//%d"
        if (q + 1 < end && q[1] == '/')
        {
            const char* u = q + 2;
            if (scan_int(u, end, c))
            {
                p = a;
                t = 0;
                n = c;
                return true;
            }
        }
        // "%d/%d"
        const char* r2 = q + 1;
        if (scan_int(r2, end, b))
        {
            p = a;
            t = b;
            n = 0;
            return true;
        }
    }
    // "%d"
    q = s;
    if (scan_int(q, end, a))
    {
        p = a;
        t = 0;
        n = 0;
        return true;
    }
    return false;
}

struct Face
{
    long long corner;   // first corner in Chunk::corners (3 ints each)
    int count;          // corners of the face
    int nv, nvt, nvn;   // chunk-local list sizes when the face was read
    int mtl;            // chunk-local usemtl event before the face, -1: inherited
};

struct Chunk
{
    const char* begin = nullptr;
    const char* end = nullptr;
    std::vector<float> v, vn, vt;
    std::vector<int> corners;
    std::vector<Face> faces;
    std::vector<std::string> mtls;
    bool faceBeforeMtl = false;
    std::string error;      // first parse error of the chunk
    // pass 2
    long long vBase = 0, vtBase = 0, vnBase = 0;
    int inherited = -1;
    std::vector<int> mtlIds;
    // pass 3
    long long triCount = 0, degenerate = 0, triBase = 0;
    std::string refError;
};

void parse_chunk(Chunk& c)
{
    // capacity guesses from the chunk size (a face or vertex line is >= 8 bytes)
    const size_t lines = (size_t)(c.end - c.begin) / 16 + 16;
    c.v.reserve(3 * lines);
    c.corners.reserve(3 * lines);
    c.faces.reserve(lines);
    const char* s = c.begin;
    while (s < c.end)
    {
        const char* eol = static_cast<const char*>(std::memchr(s, '\n', (size_t)(c.end - s)));
        if (!eol) eol = c.end;
        const char* h = s;
        while (h < eol && is_ws(*h)) ++h;
        const char* he = h;
        while (he < eol && !is_ws(*he)) ++he;
        const size_t hl = (size_t)(he - h);
        const char* rest = he;
        s = eol + 1;
        if (hl == 0) continue;
        if (hl == 1 && h[0] == 'v')
        {
            float x, y, z;
            if (!(scan_float(rest, eol, x) && scan_float(rest, eol, y) && scan_float(rest, eol, z)))
            {
                c.error = "Invalid vertex position";
                return;
            }
            c.v.push_back(x);
            c.v.push_back(y);
            c.v.push_back(z);
        }
        else if (hl == 2 && h[0] == 'v' && h[1] == 'n')
        {
            float x, y, z;
            if (!(scan_float(rest, eol, x) && scan_float(rest, eol, y) && scan_float(rest, eol, z)))
            {
                c.error = "Invalid vertex normal";
                return;
            }
            c.vn.push_back(x);
            c.vn.push_back(y);
            c.vn.push_back(z);
        }
        else if (hl == 2 && h[0] == 'v' && h[1] == 't')
        {
            float x, y;
            if (!(scan_float(rest, eol, x) && scan_float(rest, eol, y)))
            {
                c.error = "Invalid vertex texture coordinates";
                return;
            }
            c.vt.push_back(x);
            c.vt.push_back(y);
        }
        else if (hl == 1 && h[0] == 'f')
        {
            Face f;
            f.corner = (long long)c.corners.size() / 3;
            f.count = 0;
            f.nv = (int)(c.v.size() / 3);
            f.nvt = (int)(c.vt.size() / 2);
            f.nvn = (int)(c.vn.size() / 3);
            f.mtl = (int)c.mtls.size() - 1;
            const char* t = rest;
            bool ok = true;
            while (t < eol)
            {
                while (t < eol && is_face_delim(*t)) ++t;
                if (t >= eol) break;
                const char* te = t;
                while (te < eol && !is_face_delim(*te)) ++te;
                int p = 0, tx = 0, n = 0;
                if (!scan_corner(t, te, p, tx, n)) ok = false;
                c.corners.push_back(p);
                c.corners.push_back(tx);
                c.corners.push_back(n);
                ++f.count;
                t = te;
            }
            if (!ok || f.count < 3)
            {
                c.error = "Invalid face";
                return;
            }
            if (c.mtls.empty()) c.faceBeforeMtl = true;
            c.faces.push_back(f);
        }
        else if (hl == 6 && std::memcmp(h, "usemtl", 6) == 0)
        {
            const char* n = rest;
            while (n < eol && is_ws(*n)) ++n;
            const char* ne = n;
            while (ne < eol && !is_ws(*ne)) ++ne;
            if (ne == n)
            {
                c.error = "Invalid material";
                return;
            }
            c.mtls.emplace_back(n, (size_t)(ne - n));
        }
    }
}

// convertIndex (obj_loader.cpp:246-251)
inline long long convert_index(int i, long long size) { return i >= 0 ? (long long)i : (long long)i + size + 1; }

// Pass 3: one sweep counts (out == nullptr), the second writes.
// Pass 3: one sweep counts (corners == nullptr), the second writes each kept
// triangle's 0-based corner indices (position only, or position, texcoord and
// normal with -1 for none) and material id.
void emit_chunk(Chunk& c, long long nv, long long nvt, long long nvn, int cornerInts, int* corners, int* mats)
{
    long long tri = 0, degenerate = 0;
    for (const Face& f : c.faces)
    {
        const int* cr = &c.corners[3 * (size_t)f.corner];
        const int mat = f.mtl >= 0 ? c.mtlIds[(size_t)f.mtl] : c.inherited;
        long long P[3], T[3], N[3];
        auto resolve = [&](int k, int slot) {
            P[slot] = convert_index(cr[3 * k + 0], c.vBase + f.nv);
            T[slot] = convert_index(cr[3 * k + 1], c.vtBase + f.nvt);
            N[slot] = convert_index(cr[3 * k + 2], c.vnBase + f.nvn);
        };
        for (int i = 0; i + 2 < f.count; ++i)
        {
            resolve(0, 0);
            resolve(i + 1, 1);
            resolve(i + 2, 2);
            if (P[0] == P[1] || P[0] == P[2] || P[1] == P[2])
            {
                ++degenerate;
                continue;
            }
            for (int k = 0; k < 3; ++k)
            {
                // makeSoup (obj_loader.cpp:262-302)
                if (P[k] < 1 || P[k] > nv || T[k] < 0 || T[k] > nvt || N[k] < 0 || N[k] > nvn)
                {
                    if (c.refError.empty()) c.refError = "Invalid vertex reference";
                    return;
                }
            }
            if (corners)
            {
                int* o = corners + (size_t)3 * cornerInts * (size_t)(c.triBase + tri);
                for (int k = 0; k < 3; ++k)
                {
                    o[cornerInts * k] = (int)(P[k] - 1);
                    if (cornerInts == 3)
                    {
                        o[3 * k + 1] = (int)(T[k] - 1);
                        o[3 * k + 2] = (int)(N[k] - 1);
                    }
                }
                mats[c.triBase + tri] = mat;
            }
            ++tri;
        }
    }
    c.triCount = tri;
    c.degenerate = degenerate;
}

template <class F>
void parallel(int n, int threads, F&& fn)
{
    if (threads <= 1 || n <= 1)
    {
        for (int i = 0; i < n; ++i) fn(i);
        return;
    }
    std::vector<std::thread> pool;
    const int t = std::min(threads, n);
    for (int w = 0; w < t; ++w)
        pool.emplace_back([&, w] {
            for (int i = w; i < n; i += t) fn(i);
        });
    for (auto& th : pool) th.join();
}

void set_err(char* err, int errlen, const std::string& msg)
{
    if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "%s", msg.c_str());
}

} // namespace

extern "C" {

int prt_soup_load_obj(const char* path, int threads, prt_soup** soupOut, char* err, int errlen)
{
    if (!path || !soupOut) return PRT_EINVAL;
    *soupOut = nullptr;
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0)
    {
        set_err(err, errlen, std::string("Could not open OBJ file: ") + path);
        return PRT_EIO;
    }
    const long long size = (long long)::lseek(fd, 0, SEEK_END);
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    std::unique_ptr<char, HugeFree> text(static_cast<char*>(huge_alloc((size_t)std::max(0LL, size) + 1)));
    bool readOk = size >= 0 && text;
    if (readOk)
    {
        // the file in parallel pieces of at least 4 MiB
        const int pieces = (int)std::max(1LL, std::min<long long>(threads, size >> 22));
        std::vector<char> ok((size_t)pieces, 1);
        parallel(pieces, pieces, [&](int i) {
            long long at = size * i / pieces, stop = size * (i + 1) / pieces;
            while (at < stop)
            {
                ssize_t got = ::pread(fd, text.get() + at, (size_t)(stop - at), (off_t)at);
                if (got <= 0)
                {
                    ok[(size_t)i] = 0;
                    return;
                }
                at += got;
            }
        });
        for (char k : ok) readOk = readOk && k;
    }
    ::close(fd);
    if (!readOk)
    {
        set_err(err, errlen, std::string("read error: ") + path);
        return PRT_EIO;
    }
    text.get()[(size_t)size] = '\0';

    const long long minChunk = 64 << 10;
    const int nChunks = (int)std::max(1LL, std::min<long long>(4LL * threads, size / minChunk));
    std::vector<Chunk> chunks((size_t)nChunks);
    {
        const char* b = text.get();
        const char* e = b + size;
        const char* at = b;
        for (int i = 0; i < nChunks; ++i)
        {
            const char* cut = i + 1 == nChunks ? e : b + (size_t)((double)size * (i + 1) / nChunks);
            if (cut < at) cut = at;
            if (cut < e)
            {
                const char* nl = static_cast<const char*>(std::memchr(cut, '\n', (size_t)(e - cut)));
                cut = nl ? nl + 1 : e;
            }
            chunks[(size_t)i].begin = at;
            chunks[(size_t)i].end = cut;
            at = cut;
        }
    }

    // pass 1
    parallel(nChunks, threads, [&](int i) { parse_chunk(chunks[(size_t)i]); });
    for (const Chunk& c : chunks)
        if (!c.error.empty())
        {
            set_err(err, errlen, c.error);
            return PRT_EIO;
        }

    // pass 2: list bases and material ids in file order
    std::unique_ptr<prt_soup> soup(new prt_soup);
    soup->names.push_back("");   // 0 is reserved for background
    int current = -1;
    long long nv = 0, nvt = 0, nvn = 0;
    for (Chunk& c : chunks)
    {
        c.vBase = nv;
        c.vtBase = nvt;
        c.vnBase = nvn;
        nv += (long long)c.v.size() / 3;
        nvt += (long long)c.vt.size() / 2;
        nvn += (long long)c.vn.size() / 3;
        if (current < 0 && c.faceBeforeMtl)
        {
            soup->names.push_back("Default");
            current = (int)soup->names.size() - 1;
        }
        c.inherited = current;
        for (const std::string& name : c.mtls)
        {
            auto it = std::find(soup->names.begin(), soup->names.end(), name);
            if (it == soup->names.end())
            {
                soup->names.push_back(name);
                current = (int)soup->names.size() - 1;
            }
            else
                current = (int)(it - soup->names.begin());
            c.mtlIds.push_back(current);
        }
    }
    if (nv > 0x7fffffffLL || nvt > 0x7fffffffLL || nvn > 0x7fffffffLL)
    {
        set_err(err, errlen, "too many vertices");
        return PRT_EIO;
    }
    std::vector<float> v((size_t)nv * 3), vt((size_t)nvt * 2), vn((size_t)nvn * 3);
    parallel(nChunks, threads, [&](int i) {
        const Chunk& c = chunks[(size_t)i];
        if (!c.v.empty()) std::memcpy(&v[(size_t)c.vBase * 3], c.v.data(), c.v.size() * 4);
        if (!c.vt.empty()) std::memcpy(&vt[(size_t)c.vtBase * 2], c.vt.data(), c.vt.size() * 4);
        if (!c.vn.empty()) std::memcpy(&vn[(size_t)c.vnBase * 3], c.vn.data(), c.vn.size() * 4);
    });

    // pass 3: count, then write at each chunk's offset
    parallel(nChunks, threads, [&](int i) { emit_chunk(chunks[(size_t)i], nv, nvt, nvn, 1, nullptr, nullptr); });
    long long total = 0, degenerate = 0;
    for (Chunk& c : chunks)
    {
        if (!c.refError.empty())
        {
            set_err(err, errlen, c.refError);
            return PRT_EIO;
        }
        c.triBase = total;
        total += c.triCount;
        degenerate += c.degenerate;
    }
    if (total > 0x7fffffffLL / 3)
    {
        set_err(err, errlen, "too many triangles");
        return PRT_EIO;
    }
    const int cornerInts = (nvt == 0 && nvn == 0) ? 1 : 3;
    soup->corners.reset(static_cast<int*>(huge_alloc(sizeof(int) * 3 * cornerInts * (size_t)total)));
    soup->mat.reset(static_cast<int*>(huge_alloc(sizeof(int) * (size_t)total)));
    if (!soup->corners || !soup->mat)
    {
        set_err(err, errlen, "out of host memory");
        return PRT_EIO;
    }
    soup->cornerInts = cornerInts;
    soup->triCount = total;
    soup->degenerate = degenerate;
    parallel(nChunks, threads, [&](int i) {
        emit_chunk(chunks[(size_t)i], nv, nvt, nvn, cornerInts, soup->corners.get(), soup->mat.get());
    });
    soup->v = std::move(v);
    soup->vt = std::move(vt);
    soup->vn = std::move(vn);
    *soupOut = soup.release();
    return PRT_OK;
}

int prt_soup_info(const prt_soup* soup, int* triCount, int* materialCount, int* degenerateCount)
{
    if (!soup) return PRT_EINVAL;
    if (triCount) *triCount = (int)soup->triCount;
    if (materialCount) *materialCount = (int)soup->names.size();
    if (degenerateCount) *degenerateCount = (int)std::min<long long>(soup->degenerate, 0x7fffffffLL);
    return PRT_OK;
}

const prt_soup_triangle* prt_soup_triangles(const prt_soup* soup)
{
    if (!soup) return nullptr;
    prt_soup* s = const_cast<prt_soup*>(soup);   // the expansion is a cache of the indexed form
    if (!s->tris && s->triCount > 0)
    {
        std::unique_ptr<prt_soup_triangle, HugeFree> t(
            static_cast<prt_soup_triangle*>(huge_alloc(sizeof(prt_soup_triangle) * (size_t)s->triCount)));
        if (!t) return nullptr;
        const int threads = (int)std::max(1u, std::thread::hardware_concurrency());
        const long long n = s->triCount;
        const int parts = (int)std::max(1LL, std::min<long long>(4LL * threads, n / 4096));
        parallel(parts, threads, [&](int i) {
            const long long b = n * i / parts, e = n * (i + 1) / parts;
            const int ci = s->cornerInts;
            for (long long k = b; k < e; ++k)
            {
                prt_soup_triangle& o = t.get()[k];
                const int* c = s->corners.get() + (size_t)3 * ci * (size_t)k;
                for (int j = 0; j < 3; ++j)
                {
                    std::memcpy(o.v[j].pos, s->v.data() + 3 * (size_t)c[ci * j], 12);
                    const int tx = ci == 3 ? c[3 * j + 1] : -1, nr = ci == 3 ? c[3 * j + 2] : -1;
                    if (nr >= 0) std::memcpy(o.v[j].normal, s->vn.data() + 3 * (size_t)nr, 12);
                    else std::memset(o.v[j].normal, 0, 12);
                    if (tx >= 0) std::memcpy(o.v[j].tex, s->vt.data() + 2 * (size_t)tx, 8);
                    else std::memset(o.v[j].tex, 0, 8);
                }
                o.matId = s->mat.get()[k];
            }
        });
        s->tris = std::move(t);
    }
    return s->tris.get();
}

const char* prt_soup_material_name(const prt_soup* soup, int i)
{
    if (!soup || i < 0 || i >= (int)soup->names.size()) return nullptr;
    return soup->names[(size_t)i].c_str();
}

void prt_soup_free(prt_soup* soup) { delete soup; }

} // extern "C"

bool prt_b200::soup_indexed(const prt_soup* s, SoupIndexed* out)
{
    if (!s || !out) return false;
    out->v = s->v.data();
    out->nv = (long long)s->v.size() / 3;
    out->vt = s->vt.data();
    out->nvt = (long long)s->vt.size() / 2;
    out->vn = s->vn.data();
    out->nvn = (long long)s->vn.size() / 3;
    out->corners = s->corners.get();
    out->cornerInts = s->cornerInts;
    out->mat = s->mat.get();
    out->triCount = s->triCount;
    return true;
}
