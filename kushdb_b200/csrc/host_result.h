// Host-side result table and the reference's text output format.
//
// A query result is a set of typed columns.  Text formatting follows the
// reference printer (runtime/printer.cc:13-36): every value is followed by
// '|', NULL prints as an empty field, BOOLEAN as t/f, DATE through SplitDate
// as YYYY-MM-DD, REAL with std::fixed (6 decimals), ENUM as its dictionary
// string.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "plan.h"

namespace kdb {

// runtime::Date::BuildDate (runtime/date.cc:10-25): civil date -> Julian day.
inline int32_t BuildDate(int32_t year, int32_t month, int32_t day) {
  uint32_t y = static_cast<uint32_t>(year), m = static_cast<uint32_t>(month);
  if (m > 2) {
    m += 1;
    y += 4800;
  } else {
    m += 13;
    y += 4799;
  }
  int32_t century = static_cast<int32_t>(y / 100);
  int32_t julian = static_cast<int32_t>(y * 365 - 32167);
  julian += static_cast<int32_t>(y / 4) - century + century / 4;
  julian += static_cast<int32_t>(7834 * m / 256 + static_cast<uint32_t>(day));
  return julian;
}

// runtime::Date::SplitDate (runtime/date.cc:29-44): Julian day -> civil date.
inline void SplitDate(int32_t jd, int32_t* year, int32_t* month, int32_t* day) {
  uint32_t julian = static_cast<uint32_t>(jd);
  julian += 32044;
  uint32_t quad = julian / 146097;
  uint32_t extra = (julian - quad * 146097) * 4 + 3;
  julian += 60 + quad * 3 + extra / 146097;
  quad = julian / 1461;
  julian -= quad * 1461;
  int32_t y = static_cast<int32_t>(julian * 4 / 1461);
  julian = ((y != 0) ? ((julian + 305) % 365) : ((julian + 306) % 366)) + 123;
  y += static_cast<int32_t>(quad * 4);
  *year = y - 4800;
  quad = julian * 2141 / 65536;
  *day = static_cast<int32_t>(julian - 7834 * quad / 256);
  *month = static_cast<int32_t>((quad + 10) % 12 + 1);
}

inline int32_t ExtractYear(int32_t jd) {
  int32_t y, m, d;
  SplitDate(jd, &y, &m, &d);
  return y;
}

struct HostColumn {
  std::string name;
  plan::Type type;
  std::vector<int64_t> i;        // SMALLINT/INT/BIGINT/DATE/ENUM/BOOLEAN
  std::vector<double> f;         // REAL
  std::vector<std::string> s;    // TEXT
  std::vector<int8_t> null;      // 1 = NULL
  // Packed form of a downloaded non-TEXT column (the vectors above stay
  // empty): `width`-byte values as stored on the device (signed integers,
  // REAL as double) at `data`, one NULL byte per row at `nulls` (nullptr:
  // no NULLs).  The bytes belong to HostResult::block.
  bool packed = false;
  const char* data = nullptr;
  const int8_t* nulls = nullptr;
  int width = 0;

  bool IsNull(int64_t r) const { return packed ? (nulls != nullptr && nulls[r] != 0) : null[r] != 0; }
  int64_t IntAt(int64_t r) const {
    if (!packed) return i[r];
    switch (width) {
      case 1: return reinterpret_cast<const int8_t*>(data)[r];
      case 2: return reinterpret_cast<const int16_t*>(data)[r];
      case 4: return reinterpret_cast<const int32_t*>(data)[r];
      default: return reinterpret_cast<const int64_t*>(data)[r];
    }
  }
  double RealAt(int64_t r) const { return packed ? reinterpret_cast<const double*>(data)[r] : f[r]; }

  // Whole-column copies (the C interface); false when the column has no
  // values of that kind (integers of a REAL or TEXT column, reals of a
  // non-REAL column).
  bool CopyInts(int64_t rows, int64_t* out) const {
    if (!packed) {
      if (i.size() != static_cast<size_t>(rows)) return false;
      if (rows) std::memcpy(out, i.data(), sizeof(int64_t) * rows);
      return true;
    }
    if (type.id == plan::TypeId::REAL) return rows == 0;
    auto widen = [&](auto tag) {  // one tight loop per stored width
      using T = decltype(tag);
      const T* v = reinterpret_cast<const T*>(data);
      for (int64_t r = 0; r < rows; r++) out[r] = v[r];
    };
    switch (width) {
      case 1: widen(int8_t{}); break;
      case 2: widen(int16_t{}); break;
      case 4: widen(int32_t{}); break;
      default:
        if (rows) std::memcpy(out, data, sizeof(int64_t) * rows);
        break;
    }
    return true;
  }
  bool CopyReals(int64_t rows, double* out) const {
    if (!packed) {
      if (f.size() != static_cast<size_t>(rows)) return false;
      if (rows) std::memcpy(out, f.data(), sizeof(double) * rows);
      return true;
    }
    if (type.id != plan::TypeId::REAL) return rows == 0;
    if (rows) std::memcpy(out, data, sizeof(double) * rows);
    return true;
  }
  void CopyNulls(int64_t rows, int8_t* out) const {
    if (!packed) {
      if (!null.empty()) std::memcpy(out, null.data(), null.size());
    } else if (nulls) {
      std::memcpy(out, nulls, rows);
    } else if (rows) {
      std::memset(out, 0, rows);
    }
  }
};

struct HostResult {
  std::vector<HostColumn> cols;
  int64_t rows = 0;
  std::shared_ptr<char> block;  // owns the packed columns' bytes
};

using EnumDicts = std::map<int32_t, std::vector<std::string>>;

inline std::string FormatValue(const HostColumn& c, int64_t r, const EnumDicts& enums) {
  if (c.IsNull(r)) return "";
  char buf[64];
  switch (c.type.id) {
    case plan::TypeId::BOOLEAN: return c.IntAt(r) ? "t" : "f";
    case plan::TypeId::SMALLINT:
    case plan::TypeId::INT:
    case plan::TypeId::BIGINT:
      std::snprintf(buf, sizeof(buf), "%lld", static_cast<long long>(c.IntAt(r)));
      return buf;
    case plan::TypeId::DATE: {
      int32_t y, m, d;
      SplitDate(static_cast<int32_t>(c.IntAt(r)), &y, &m, &d);
      std::snprintf(buf, sizeof(buf), "%d-%02d-%02d", y, m, d);
      return buf;
    }
    case plan::TypeId::REAL:
      std::snprintf(buf, sizeof(buf), "%.6f", c.RealAt(r));
      return buf;
    case plan::TypeId::TEXT: return c.s[r];
    case plan::TypeId::ENUM: {
      auto it = enums.find(c.type.enum_id);
      int64_t k = c.IntAt(r);
      if (it == enums.end() || k < 0 || k >= static_cast<int64_t>(it->second.size()))
        return "<enum:" + std::to_string(k) + ">";
      return it->second[k];
    }
  }
  return "";
}

// One line per row, "v|v|...|\n" (runtime/printer.cc).
inline std::string FormatResult(const HostResult& res, const EnumDicts& enums) {
  std::string out;
  for (int64_t r = 0; r < res.rows; r++) {
    for (const auto& c : res.cols) {
      out += FormatValue(c, r, enums);
      out += '|';
    }
    out += '\n';
  }
  return out;
}

}  // namespace kdb
