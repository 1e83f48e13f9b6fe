// Project-written stand-in for the subset of the mp-units 2.4 API that the
// Lucid reference headers use (LucidRenderer/cpp_renderer/include/units/
// render_units.hpp and the headers that include it).  TEST INFRASTRUCTURE:
// it exists only so that the reference's own C++ render path can be compiled
// here (mp-units is not installed) and run beside the oracle as its pin and as
// the timed CPU baseline.
//
// Every unit the reference uses has magnitude 1 (metre, square metre, watt,
// radian, steradian, one), so a quantity is its number plus compile-time
// bookkeeping: arithmetic is the plain arithmetic of the representation type
// in the order the expression states, exactly as mp-units compiles it.
//
// Design (not mp-units' own): a unit is a type carrying four exponents
// (length, power, plane angle, solid angle); a reference pairs a quantity-kind
// tag with a unit; quantity<R, Rep> holds one Rep.  Conversions between
// quantities are implicit whenever the unit exponents agree (a superset of
// what mp-units accepts, which is enough to compile correct code; the
// reference's static_asserts on exact result types still hold because the
// reference states its result types explicitly).
#pragma once

#include <cmath>
#include <compare>
#include <concepts>
#include <type_traits>
#include <utility>

namespace mp_units {

// ---------------------------------------------------------------- customisation points
template <class T>
inline constexpr bool is_vector = false;
template <class T>
inline constexpr bool is_scalar = std::is_arithmetic_v<T>;

enum class quantity_character { scalar, vector, tensor };

// ---------------------------------------------------------------- units
template <int L, int P, int A, int S>
struct unit_dims {
    static constexpr int length = L, power = P, angle = A, solid_angle = S;
};

template <class U>
inline constexpr bool is_unit_v = false;
template <int L, int P, int A, int S>
inline constexpr bool is_unit_v<unit_dims<L, P, A, S>> = true;

template <int L1, int P1, int A1, int S1, int L2, int P2, int A2, int S2>
constexpr auto operator*(unit_dims<L1, P1, A1, S1>, unit_dims<L2, P2, A2, S2>) {
    return unit_dims<L1 + L2, P1 + P2, A1 + A2, S1 + S2>{};
}
template <int L1, int P1, int A1, int S1, int L2, int P2, int A2, int S2>
constexpr auto operator/(unit_dims<L1, P1, A1, S1>, unit_dims<L2, P2, A2, S2>) {
    return unit_dims<L1 - L2, P1 - P2, A1 - A2, S1 - S2>{};
}
template <int L, int P, int A, int S>
constexpr auto square(unit_dims<L, P, A, S>) { return unit_dims<2 * L, 2 * P, 2 * A, 2 * S>{}; }
template <int L, int P, int A, int S>
constexpr auto cubic(unit_dims<L, P, A, S>) { return unit_dims<3 * L, 3 * P, 3 * A, 3 * S>{}; }
template <int L, int P, int A, int S>
    requires(L % 2 == 0 && P % 2 == 0 && A % 2 == 0 && S % 2 == 0)
constexpr auto sqrt(unit_dims<L, P, A, S>) { return unit_dims<L / 2, P / 2, A / 2, S / 2>{}; }

inline constexpr unit_dims<0, 0, 0, 0> one{};

// ---------------------------------------------------------------- quantity kinds and references
template <class Spec, class U>
struct reference {
    using spec = Spec;
    using unit_type = U;
};

// Base of every quantity-kind tag; Self is the tag's own type.
template <class Self, auto... Args>
struct quantity_spec_base {
    template <class U>
        requires is_unit_v<U>
    constexpr reference<Self, U> operator[](U) const { return {}; }
};

// What QUANTITY_SPEC(name, parent, character...) derives from.
template <class Self, auto Parent, auto... Args>
struct quantity_spec : quantity_spec_base<Self, Parent, Args...> {};

inline constexpr struct dimensionless_ final : quantity_spec_base<dimensionless_> {
} dimensionless;

template <class R>
struct ref_traits;   // unit of a reference or of a bare unit
template <int L, int P, int A, int S>
struct ref_traits<unit_dims<L, P, A, S>> {
    using unit = unit_dims<L, P, A, S>;
};
template <class Spec, class U>
struct ref_traits<reference<Spec, U>> {
    using unit = U;
};
template <auto R>
using unit_of = typename ref_traits<std::remove_cvref_t<decltype(R)>>::unit;

template <class U1, class U2>
inline constexpr bool same_dims = std::is_same_v<U1, U2>;

// A number that may multiply or divide a quantity: arithmetic, or a vector
// representation declared through is_vector.
template <class T>
concept Representation = std::is_arithmetic_v<std::remove_cvref_t<T>> || is_vector<std::remove_cvref_t<T>>;

// ---------------------------------------------------------------- quantity
template <auto R, class Rep = double>
class quantity {
public:
    Rep numerical_value_is_an_implementation_detail_{};

    using rep = Rep;
    using unit_type = unit_of<R>;
    static constexpr auto reference = R;
    static constexpr unit_type unit{};

    quantity() = default;
    constexpr quantity(const quantity&) = default;
    constexpr quantity& operator=(const quantity&) = default;

    // quantity{value, reference}
    template <class V, class R2>
        requires std::is_convertible_v<V, Rep> && std::is_same_v<std::remove_cvref_t<R2>, std::remove_cvref_t<decltype(R)>>
    constexpr quantity(V&& v, R2) : numerical_value_is_an_implementation_detail_(std::forward<V>(v)) {}

    // a plain number is a quantity of the unit one (mp-units allows this for one only)
    template <class V>
        requires std::is_same_v<unit_type, unit_dims<0, 0, 0, 0>> && std::is_arithmetic_v<std::remove_cvref_t<V>> &&
                 std::is_convertible_v<V, Rep>
    constexpr quantity(V&& v) : numerical_value_is_an_implementation_detail_(std::forward<V>(v)) {}

    // any quantity of the same dimensions converts (all magnitudes are 1)
    template <auto R2, class Rep2>
        requires(!std::is_same_v<quantity<R2, Rep2>, quantity>) && same_dims<unit_of<R2>, unit_type> &&
                std::is_convertible_v<Rep2, Rep>
    constexpr quantity(const quantity<R2, Rep2>& q)
        : numerical_value_is_an_implementation_detail_(q.numerical_value_is_an_implementation_detail_) {}

    template <class U>
        requires same_dims<U, unit_type>
    constexpr Rep numerical_value_in(U) const {
        return numerical_value_is_an_implementation_detail_;
    }
    template <class U>
        requires same_dims<U, unit_type>
    constexpr const Rep& numerical_value_ref_in(U) const& {
        return numerical_value_is_an_implementation_detail_;
    }
    template <class U>
        requires same_dims<U, unit_type>
    constexpr Rep& numerical_value_ref_in(U) & {
        return numerical_value_is_an_implementation_detail_;
    }
    template <class U>
    void numerical_value_ref_in(U) const&& = delete;

    template <class U>
        requires same_dims<U, unit_type>
    constexpr quantity<U{}, Rep> in(U) const {
        return quantity<U{}, Rep>{numerical_value_is_an_implementation_detail_, U{}};
    }

    static constexpr quantity zero() { return quantity{}; }

    constexpr quantity operator+() const { return *this; }
    constexpr quantity operator-() const {
        quantity q;
        q.numerical_value_is_an_implementation_detail_ = -numerical_value_is_an_implementation_detail_;
        return q;
    }
    template <auto R2, class Rep2>
        requires same_dims<unit_of<R2>, unit_type>
    constexpr quantity& operator+=(const quantity<R2, Rep2>& o) {
        numerical_value_is_an_implementation_detail_ += o.numerical_value_is_an_implementation_detail_;
        return *this;
    }
    template <auto R2, class Rep2>
        requires same_dims<unit_of<R2>, unit_type>
    constexpr quantity& operator-=(const quantity<R2, Rep2>& o) {
        numerical_value_is_an_implementation_detail_ -= o.numerical_value_is_an_implementation_detail_;
        return *this;
    }
    template <class V>
        requires std::is_arithmetic_v<V>
    constexpr quantity& operator*=(V s) {
        numerical_value_is_an_implementation_detail_ *= s;
        return *this;
    }
    template <class V>
        requires std::is_arithmetic_v<V>
    constexpr quantity& operator/=(V s) {
        numerical_value_is_an_implementation_detail_ /= s;
        return *this;
    }
};

template <class V, class R>
quantity(V, R) -> quantity<R{}, std::remove_cvref_t<V>>;

template <class T>
inline constexpr bool is_quantity_v = false;
template <auto R, class Rep>
inline constexpr bool is_quantity_v<quantity<R, Rep>> = true;

namespace detail {
template <auto R, class Rep>
constexpr const Rep& val(const quantity<R, Rep>& q) { return q.numerical_value_is_an_implementation_detail_; }
template <auto R, class Rep>
constexpr quantity<R, Rep> make(Rep v) {
    quantity<R, Rep> q;
    q.numerical_value_is_an_implementation_detail_ = v;
    return q;
}
}  // namespace detail

// number * unit, unit * number -> quantity of that unit
template <class V, int L, int P, int A, int S>
    requires Representation<V>
constexpr auto operator*(V&& v, unit_dims<L, P, A, S>) {
    return detail::make<unit_dims<L, P, A, S>{}, std::remove_cvref_t<V>>(v);
}
template <class V, int L, int P, int A, int S>
    requires Representation<V>
constexpr auto operator/(V&& v, unit_dims<L, P, A, S>) {
    return detail::make<unit_dims<-L, -P, -A, -S>{}, std::remove_cvref_t<V>>(v);
}

// quantity * unit, quantity / unit
template <auto R, class Rep, int L, int P, int A, int S>
constexpr auto operator*(const quantity<R, Rep>& q, unit_dims<L, P, A, S> u) {
    return detail::make<unit_of<R>{} * u, Rep>(detail::val(q));
}
template <auto R, class Rep, int L, int P, int A, int S>
constexpr auto operator/(const quantity<R, Rep>& q, unit_dims<L, P, A, S> u) {
    return detail::make<unit_of<R>{} / u, Rep>(detail::val(q));
}

// quantity (+|-) quantity
template <auto R1, class Rep1, auto R2, class Rep2>
    requires same_dims<unit_of<R1>, unit_of<R2>>
constexpr auto operator+(const quantity<R1, Rep1>& a, const quantity<R2, Rep2>& b) {
    using Rep = decltype(detail::val(a) + detail::val(b));
    if constexpr (std::is_same_v<quantity<R1, Rep1>, quantity<R2, Rep2>> && std::is_same_v<Rep, Rep1>)
        return detail::make<R1, Rep>(detail::val(a) + detail::val(b));
    else
        return detail::make<unit_of<R1>{}, Rep>(detail::val(a) + detail::val(b));
}
template <auto R1, class Rep1, auto R2, class Rep2>
    requires same_dims<unit_of<R1>, unit_of<R2>>
constexpr auto operator-(const quantity<R1, Rep1>& a, const quantity<R2, Rep2>& b) {
    using Rep = decltype(detail::val(a) - detail::val(b));
    if constexpr (std::is_same_v<quantity<R1, Rep1>, quantity<R2, Rep2>> && std::is_same_v<Rep, Rep1>)
        return detail::make<R1, Rep>(detail::val(a) - detail::val(b));
    else
        return detail::make<unit_of<R1>{}, Rep>(detail::val(a) - detail::val(b));
}

// quantity (*|/) quantity
template <auto R1, class Rep1, auto R2, class Rep2>
constexpr auto operator*(const quantity<R1, Rep1>& a, const quantity<R2, Rep2>& b) {
    using Rep = decltype(detail::val(a) * detail::val(b));
    return detail::make<unit_of<R1>{} * unit_of<R2>{}, Rep>(detail::val(a) * detail::val(b));
}
template <auto R1, class Rep1, auto R2, class Rep2>
constexpr auto operator/(const quantity<R1, Rep1>& a, const quantity<R2, Rep2>& b) {
    using Rep = decltype(detail::val(a) / detail::val(b));
    return detail::make<unit_of<R1>{} / unit_of<R2>{}, Rep>(detail::val(a) / detail::val(b));
}

// number (*|/) quantity, quantity (*|/) number
template <class V, auto R, class Rep>
    requires Representation<V>
constexpr auto operator*(const V& s, const quantity<R, Rep>& q) {
    using Out = decltype(s * detail::val(q));
    return detail::make<R, Out>(s * detail::val(q));
}
template <auto R, class Rep, class V>
    requires Representation<V>
constexpr auto operator*(const quantity<R, Rep>& q, const V& s) {
    using Out = decltype(detail::val(q) * s);
    return detail::make<R, Out>(detail::val(q) * s);
}
template <auto R, class Rep, class V>
    requires Representation<V>
constexpr auto operator/(const quantity<R, Rep>& q, const V& s) {
    using Out = decltype(detail::val(q) / s);
    return detail::make<R, Out>(detail::val(q) / s);
}
template <class V, auto R, class Rep>
    requires std::is_arithmetic_v<V>
constexpr auto operator/(const V& s, const quantity<R, Rep>& q) {
    using Out = decltype(s / detail::val(q));
    return detail::make<unit_dims<0, 0, 0, 0>{} / unit_of<R>{}, Out>(s / detail::val(q));
}

// comparisons between quantities of the same dimensions
template <auto R1, class Rep1, auto R2, class Rep2>
    requires same_dims<unit_of<R1>, unit_of<R2>>
constexpr bool operator==(const quantity<R1, Rep1>& a, const quantity<R2, Rep2>& b) {
    return detail::val(a) == detail::val(b);
}
template <auto R1, class Rep1, auto R2, class Rep2>
    requires same_dims<unit_of<R1>, unit_of<R2>> && std::is_arithmetic_v<Rep1> && std::is_arithmetic_v<Rep2>
constexpr auto operator<=>(const quantity<R1, Rep1>& a, const quantity<R2, Rep2>& b) {
    return detail::val(a) <=> detail::val(b);
}

template <auto R, class Rep>
    requires std::is_arithmetic_v<Rep>
constexpr quantity<R, Rep> abs(const quantity<R, Rep>& q) {
    return detail::make<R, Rep>(q.numerical_value_is_an_implementation_detail_ < Rep(0)
                                    ? -q.numerical_value_is_an_implementation_detail_
                                    : q.numerical_value_is_an_implementation_detail_);
}

// ---------------------------------------------------------------- affine points
template <auto QS>
struct absolute_point_origin {
    static constexpr auto quantity_spec = QS;
};

template <class T>
concept PointOrigin = requires { T::quantity_spec; } && std::is_empty_v<T>;

template <auto R, auto PO, class Rep = double>
class quantity_point {
public:
    quantity<R, Rep> quantity_from_origin_is_an_implementation_detail_{};

    using rep = Rep;
    using quantity_type = quantity<R, Rep>;
    static constexpr auto reference = R;
    static constexpr auto point_origin = PO;

    quantity_point() = default;
    constexpr explicit quantity_point(const quantity_type& q) : quantity_from_origin_is_an_implementation_detail_(q) {}
    constexpr quantity_point(const quantity_type& q, std::remove_cvref_t<decltype(PO)>)
        : quantity_from_origin_is_an_implementation_detail_(q) {}

    template <class O>
        requires std::is_same_v<O, std::remove_cvref_t<decltype(PO)>>
    constexpr quantity_type quantity_from(O) const {
        return quantity_from_origin_is_an_implementation_detail_;
    }
    constexpr const quantity_type& quantity_ref_from(std::remove_cvref_t<decltype(PO)>) const& {
        return quantity_from_origin_is_an_implementation_detail_;
    }
    constexpr quantity_type quantity_from_zero() const { return quantity_from_origin_is_an_implementation_detail_; }

    template <auto R2, class Rep2>
        requires same_dims<unit_of<R2>, unit_of<R>>
    constexpr quantity_point& operator+=(const quantity<R2, Rep2>& q) {
        quantity_from_origin_is_an_implementation_detail_ += q;
        return *this;
    }
    template <auto R2, class Rep2>
        requires same_dims<unit_of<R2>, unit_of<R>>
    constexpr quantity_point& operator-=(const quantity<R2, Rep2>& q) {
        quantity_from_origin_is_an_implementation_detail_ -= q;
        return *this;
    }

    friend constexpr bool operator==(const quantity_point& a, const quantity_point& b) {
        return a.quantity_from_origin_is_an_implementation_detail_ == b.quantity_from_origin_is_an_implementation_detail_;
    }
};

// origin + quantity -> point
template <class O, auto R, class Rep>
    requires PointOrigin<O>
constexpr auto operator+(O, const quantity<R, Rep>& q) {
    return quantity_point<R, O{}, Rep>(q);
}
template <auto R, class Rep, class O>
    requires PointOrigin<O>
constexpr auto operator+(const quantity<R, Rep>& q, O) {
    return quantity_point<R, O{}, Rep>(q);
}

// point +/- quantity -> point; point - point -> quantity
template <auto R, auto PO, class Rep, auto R2, class Rep2>
    requires same_dims<unit_of<R2>, unit_of<R>>
constexpr quantity_point<R, PO, Rep> operator+(const quantity_point<R, PO, Rep>& p, const quantity<R2, Rep2>& q) {
    return quantity_point<R, PO, Rep>(quantity<R, Rep>(p.quantity_from_origin_is_an_implementation_detail_ + q));
}
template <auto R, auto PO, class Rep, auto R2, class Rep2>
    requires same_dims<unit_of<R2>, unit_of<R>>
constexpr quantity_point<R, PO, Rep> operator+(const quantity<R2, Rep2>& q, const quantity_point<R, PO, Rep>& p) {
    return quantity_point<R, PO, Rep>(quantity<R, Rep>(q + p.quantity_from_origin_is_an_implementation_detail_));
}
template <auto R, auto PO, class Rep, auto R2, class Rep2>
    requires same_dims<unit_of<R2>, unit_of<R>>
constexpr quantity_point<R, PO, Rep> operator-(const quantity_point<R, PO, Rep>& p, const quantity<R2, Rep2>& q) {
    return quantity_point<R, PO, Rep>(quantity<R, Rep>(p.quantity_from_origin_is_an_implementation_detail_ - q));
}
template <auto R, auto PO, class Rep>
constexpr quantity<R, Rep> operator-(const quantity_point<R, PO, Rep>& a, const quantity_point<R, PO, Rep>& b) {
    return a.quantity_from_origin_is_an_implementation_detail_ - b.quantity_from_origin_is_an_implementation_detail_;
}

}  // namespace mp_units
