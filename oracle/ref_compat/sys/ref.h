// Reference-counted pointer with the interface ProtoRay's renderer code uses
// (ref<T>, makeRef, staticRefCast, dynamicRefCast; reference: sys/ref.h:30-223).
//
// Test infrastructure only: this header lets GCC compile the reference's own
// CPU renderer from its unmodified sources (the original header declares
// friend templates whose parameter shadows the class parameter, which GCC
// rejects). It sits earlier on the include path than the reference tree and
// is built on std::shared_ptr; nothing in the product links it.
#pragma once

#include <cstddef>
#include <memory>
#include <utility>

namespace prt {

template <class T>
class ref
{
    template <class U> friend class ref;
    std::shared_ptr<T> p;

public:
    ref() = default;
    ref(std::nullptr_t) {}
    explicit ref(std::shared_ptr<T> sp) : p(std::move(sp)) {}
    template <class U> ref(const ref<U>& o) : p(o.p) {}

    T* get() const { return p.get(); }
    T* operator->() const { return p.get(); }
    T& operator*() const { return *p; }
    explicit operator bool() const { return bool(p); }
    bool operator!() const { return !p; }
    template <class U> bool operator==(const ref<U>& o) const { return p == o.p; }
    template <class U> bool operator!=(const ref<U>& o) const { return p != o.p; }
    bool operator==(std::nullptr_t) const { return !p; }
    bool operator!=(std::nullptr_t) const { return bool(p); }

    const std::shared_ptr<T>& shared() const { return p; }
};

template <class T, class... Args>
inline ref<T> makeRef(Args&&... args)
{
    return ref<T>(std::make_shared<T>(std::forward<Args>(args)...));
}

template <class T1, class T2>
inline ref<T1> staticRefCast(const ref<T2>& r)
{
    return ref<T1>(std::static_pointer_cast<T1>(r.shared()));
}

template <class T1, class T2>
inline ref<T1> dynamicRefCast(const ref<T2>& r)
{
    return ref<T1>(std::dynamic_pointer_cast<T1>(r.shared()));
}

} // namespace prt
