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
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/prt_b200.h"

struct prt_soup
{
    std::unique_ptr<prt_soup_triangle[]> tris;
    long long triCount = 0;
    std::vector<std::string> names;
    long long degenerate = 0;
};

namespace {

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f' || c == '\n'; }
// strtok delimiters of the face parser (obj_loader.cpp:163)
inline bool is_face_delim(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }

// sscanf "%f": skips white space, then strtof.  `end` bounds the line.
bool scan_float(const char*& s, const char* end, float& out)
{
    while (s < end && is_ws(*s)) ++s;
    if (s >= end) return false;
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
    // "%d/%d/%d"
    if (scan_int(q, end, a) && q < end && *q == '/')
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
            c.v.insert(c.v.end(), {x, y, z});
        }
        else if (hl == 2 && h[0] == 'v' && h[1] == 'n')
        {
            float x, y, z;
            if (!(scan_float(rest, eol, x) && scan_float(rest, eol, y) && scan_float(rest, eol, z)))
            {
                c.error = "Invalid vertex normal";
                return;
            }
            c.vn.insert(c.vn.end(), {x, y, z});
        }
        else if (hl == 2 && h[0] == 'v' && h[1] == 't')
        {
            float x, y;
            if (!(scan_float(rest, eol, x) && scan_float(rest, eol, y)))
            {
                c.error = "Invalid vertex texture coordinates";
                return;
            }
            c.vt.insert(c.vt.end(), {x, y});
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
                c.corners.insert(c.corners.end(), {p, tx, n});
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
void emit_chunk(Chunk& c, long long nv, long long nvt, long long nvn, const float* v, const float* vt, const float* vn,
                prt_soup_triangle* out)
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
            if (out)
            {
                prt_soup_triangle& o = out[c.triBase + tri];
                for (int k = 0; k < 3; ++k)
                {
                    std::memcpy(o.v[k].pos, v + 3 * (P[k] - 1), 12);
                    if (N[k]) std::memcpy(o.v[k].normal, vn + 3 * (N[k] - 1), 12);
                    else std::memset(o.v[k].normal, 0, 12);
                    if (T[k]) std::memcpy(o.v[k].tex, vt + 2 * (T[k] - 1), 8);
                    else std::memset(o.v[k].tex, 0, 8);
                }
                o.matId = mat;
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
    FILE* f = std::fopen(path, "rb");
    if (!f)
    {
        set_err(err, errlen, std::string("Could not open OBJ file: ") + path);
        return PRT_EIO;
    }
    std::fseek(f, 0, SEEK_END);
    const long long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::unique_ptr<char[]> text(new char[(size_t)size + 1]);
    const bool readOk = size >= 0 && std::fread(text.get(), 1, (size_t)size, f) == (size_t)size;
    std::fclose(f);
    if (!readOk)
    {
        set_err(err, errlen, std::string("read error: ") + path);
        return PRT_EIO;
    }
    text[(size_t)size] = '\0';

    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
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
    parallel(nChunks, threads,
             [&](int i) { emit_chunk(chunks[(size_t)i], nv, nvt, nvn, v.data(), vt.data(), vn.data(), nullptr); });
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
    soup->tris.reset(new prt_soup_triangle[(size_t)std::max(1LL, total)]);
    soup->triCount = total;
    soup->degenerate = degenerate;
    parallel(nChunks, threads, [&](int i) {
        emit_chunk(chunks[(size_t)i], nv, nvt, nvn, v.data(), vt.data(), vn.data(), soup->tris.get());
    });
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

const prt_soup_triangle* prt_soup_triangles(const prt_soup* soup) { return soup ? soup->tris.get() : nullptr; }

const char* prt_soup_material_name(const prt_soup* soup, int i)
{
    if (!soup || i < 0 || i >= (int)soup->names.size()) return nullptr;
    return soup->names[(size_t)i].c_str();
}

void prt_soup_free(prt_soup* soup) { delete soup; }

} // extern "C"
