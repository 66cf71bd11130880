"""The build-time annotation step (CPU): what it marks and what it leaves alone."""
from cospanmdao_b200.annotate import HD, annotate_text


def test_marks_bodies_helpers_and_device_lambdas():
    src = """
    static void compute_forward(cs::GroupItem<1> it, const Inputs& in, const Outputs& out) {}
inline std::uint32_t u32(std::size_t v) { return v; }
template <class T> inline T tmin(T a, T b) { return a < b ? a : b; }
    template <class T> static T slope(T a, T b) { return a; }
inline std::vector<std::int32_t> geo_values(int nx, int ny) { return {}; }
auto make_init(int nx, int ny, float amp) {
    return cs::init::custom<DType::f32, 3>([](auto&...) {
        return q.parallel_for(dev, deps, sycl::range<1>{n}, [=](sycl::id<1> t) { });
    });
}
"""
    out = annotate_text(src)
    assert HD + "static void compute_forward(" in out
    assert HD + "inline std::uint32_t u32(" in out
    assert "template <class T> " + HD + "inline T tmin(" in out
    assert HD + "static T slope(" in out
    assert "inline std::vector<std::int32_t> geo_values(" in out and HD + "inline std::vector" not in out
    assert "[=] " + HD + "(sycl::id<1> t)" in out
    assert "naga::cospan::InitSpec make_init(" in out
    # idempotent
    assert annotate_text(out) == out
