// Reads "op a b" lines (decimal operands) from stdin and prints one result per
// line, using the in-repo ZZ of include/cuPoly/zz.h.  tests/test_cxx_host.py
// checks every line against Python's integers.
//   ops: add sub mul div mod (floor, sign of the divisor, as NTL) shl shr (b = bit count)
//        cmp (-1 / 0 / 1) bits (NumBits of a) limbs (little-endian words of |a|, round trip)
#include <cuPoly/zz.h>

#include <iostream>
#include <sstream>
#include <string>

int main() {
  using cupoly::ZZ;
  std::string line;
  while (std::getline(std::cin, line)) {
    std::istringstream in(line);
    std::string op, sa, sb;
    in >> op >> sa >> sb;
    const ZZ a = ZZ::from_string(sa);
    const ZZ b = sb.empty() ? ZZ(0) : ZZ::from_string(sb);
    try {
      if (op == "add") std::cout << a + b;
      else if (op == "sub") std::cout << a - b;
      else if (op == "mul") std::cout << a * b;
      else if (op == "div") std::cout << a / b;
      else if (op == "mod") std::cout << a % b;
      else if (op == "shl") std::cout << (a << cupoly::to_long(b));
      else if (op == "shr") std::cout << (a >> cupoly::to_long(b));
      else if (op == "cmp") std::cout << ZZ::compare(a, b);
      else if (op == "bits") std::cout << cupoly::NumBits(a);
      else if (op == "limbs") {
        const ZZ r = ZZ::from_limbs(a.limbs().data(), a.limbs().size(), a.is_negative());
        std::cout << r;
      } else std::cout << "?";
    } catch (const std::exception& e) {
      std::cout << "error";
    }
    std::cout << "\n";
  }
  return 0;
}
