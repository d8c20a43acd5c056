/*
 * Minimal stand-in for <poplar/Vertex.hpp> — TEST INFRASTRUCTURE (oracle).
 *
 * Lets the reference's lbm_codelets.cpp compile unmodified on the host so
 * that ref_poplar_emu.cpp can run its Vertex::compute() bodies.  Only what
 * those codelets touch is provided: Vertex, Vector<T> as a pointer view and
 * the Input/Output/InOut field wrappers (scalar fields convert to T, vector
 * fields index like arrays).
 */
#pragma once
namespace poplar {

class Vertex {};

template <class T>
struct Vector {
  T* data = nullptr;
  unsigned count = 0;
  T& operator[](unsigned i) const { return data[i]; }
  unsigned size() const { return count; }
};

template <class T>
struct Input {
  T value{};
  operator const T&() const { return value; }
};
template <class T>
struct Input<Vector<T>> {
  Vector<T> value;
  const T& operator[](unsigned i) const { return value.data[i]; }
};

template <class T>
struct Output {
  T value{};
  operator T&() { return value; }
};
template <class T>
struct Output<Vector<T>> {
  Vector<T> value;
  T& operator[](unsigned i) const { return value.data[i]; }
};

template <class T>
struct InOut {
  T value{};
  operator T&() { return value; }
};
template <class T>
struct InOut<Vector<T>> {
  Vector<T> value;
  T& operator[](unsigned i) const { return value.data[i]; }
};

}  // namespace poplar
