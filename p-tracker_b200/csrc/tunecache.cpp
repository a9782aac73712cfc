// Autotune cache: the shapes ptk_autotune chose, per (GPU, workload)
// signature, in a small JSON file (host only, no CUDA), so that a run on the
// same GPU model and workload takes the stored choice instead of timing the
// candidates again.  File layout:
//
//   {"version": 1, "entries": {"<signature>": {"method": 1, "choice": 4,
//     "values": [2, 3, 4, 6], "ms": [1.46, 1.19, 1.2, 1.52]}, ...}}
//
// The reader accepts any JSON of that shape (whitespace, key order, other
// keys ignored); an entry whose fields are missing or mistyped makes the
// file malformed.  Writes replace the file through a temporary file of their
// own (named for the process and the call) and a rename, so a reader never
// sees half a file; of two writers at once, the last rename wins.
#include <unistd.h>

#include <atomic>
#include <cerrno>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "ptk.h"

namespace {

struct Entry {
  int method = 0, choice = 0;
  std::vector<int> values;
  std::vector<double> ms;
};

// Minimal recursive-descent JSON reader over the subset the cache needs:
// objects, arrays, strings (with the standard escapes), numbers, true/false/null.
struct Reader {
  const std::string& s;
  size_t i = 0;
  bool ok = true;
  explicit Reader(const std::string& text) : s(text) {}

  void ws() {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) ++i;
  }
  bool eat(char c) {
    ws();
    if (i < s.size() && s[i] == c) {
      ++i;
      return true;
    }
    return false;
  }
  bool str(std::string* out) {
    ws();
    if (i >= s.size() || s[i] != '"') return ok = false;
    ++i;
    std::string r;
    while (i < s.size() && s[i] != '"') {
      char c = s[i++];
      if (c == '\\') {
        if (i >= s.size()) return ok = false;
        const char e = s[i++];
        switch (e) {
          case '"': c = '"'; break;
          case '\\': c = '\\'; break;
          case '/': c = '/'; break;
          case 'n': c = '\n'; break;
          case 't': c = '\t'; break;
          case 'r': c = '\r'; break;
          case 'b': c = '\b'; break;
          case 'f': c = '\f'; break;
          case 'u': {  // code points below 0x80 only (the writer emits no others)
            if (i + 4 > s.size()) return ok = false;
            unsigned v = 0;
            for (int k = 0; k < 4; ++k) {
              const char h = s[i++];
              v <<= 4;
              if (h >= '0' && h <= '9') v |= (unsigned)(h - '0');
              else if (h >= 'a' && h <= 'f') v |= (unsigned)(h - 'a' + 10);
              else if (h >= 'A' && h <= 'F') v |= (unsigned)(h - 'A' + 10);
              else return ok = false;
            }
            if (v >= 0x80) return ok = false;
            c = (char)v;
            break;
          }
          default: return ok = false;
        }
      }
      r.push_back(c);
    }
    if (i >= s.size()) return ok = false;
    ++i;
    if (out) *out = r;
    return true;
  }
  bool num(double* out) {
    ws();
    const char* b = s.c_str() + i;
    char* e = nullptr;
    errno = 0;
    const double v = strtod(b, &e);
    if (e == b || errno == ERANGE) return ok = false;
    i += (size_t)(e - b);
    if (out) *out = v;
    return true;
  }
  // skips one value of any type
  bool skip() {
    ws();
    if (i >= s.size()) return ok = false;
    const char c = s[i];
    if (c == '"') return str(nullptr);
    if (c == '{') {
      ++i;
      if (eat('}')) return true;
      do {
        if (!str(nullptr) || !eat(':') || !skip()) return ok = false;
      } while (eat(','));
      return eat('}') || (ok = false);
    }
    if (c == '[') {
      ++i;
      if (eat(']')) return true;
      do {
        if (!skip()) return ok = false;
      } while (eat(','));
      return eat(']') || (ok = false);
    }
    for (const char* w : {"true", "false", "null"}) {
      const size_t n = strlen(w);
      if (s.compare(i, n, w) == 0) {
        i += n;
        return true;
      }
    }
    return num(nullptr);
  }
  bool int_array(std::vector<int>* out) {
    if (!eat('[')) return ok = false;
    out->clear();
    if (eat(']')) return true;
    do {
      double v;
      if (!num(&v)) return false;
      out->push_back((int)v);
    } while (eat(','));
    return eat(']') || (ok = false);
  }
  bool real_array(std::vector<double>* out) {
    if (!eat('[')) return ok = false;
    out->clear();
    if (eat(']')) return true;
    do {
      double v;
      if (!num(&v)) return false;
      out->push_back(v);
    } while (eat(','));
    return eat(']') || (ok = false);
  }
  bool entry(Entry* e) {
    if (!eat('{')) return ok = false;
    bool have_m = false, have_c = false;
    if (!eat('}')) {
      do {
        std::string k;
        if (!str(&k) || !eat(':')) return ok = false;
        double v;
        if (k == "method") {
          if (!num(&v)) return false;
          e->method = (int)v;
          have_m = true;
        } else if (k == "choice") {
          if (!num(&v)) return false;
          e->choice = (int)v;
          have_c = true;
        } else if (k == "values") {
          if (!int_array(&e->values)) return false;
        } else if (k == "ms") {
          if (!real_array(&e->ms)) return false;
        } else if (!skip()) {
          return false;
        }
      } while (eat(','));
      if (!eat('}')) return ok = false;
    }
    return (have_m && have_c) || (ok = false);
  }
  bool file(std::map<std::string, Entry>* out) {
    if (!eat('{')) return ok = false;
    if (eat('}')) return true;
    do {
      std::string k;
      if (!str(&k) || !eat(':')) return ok = false;
      if (k == "entries") {
        if (!eat('{')) return ok = false;
        if (!eat('}')) {
          do {
            std::string sig;
            Entry e;
            if (!str(&sig) || !eat(':') || !entry(&e)) return ok = false;
            (*out)[sig] = e;
          } while (eat(','));
          if (!eat('}')) return ok = false;
        }
      } else if (!skip()) {
        return false;
      }
    } while (eat(','));
    if (!eat('}')) return ok = false;
    ws();
    return i == s.size() || (ok = false);
  }
};

// 1 = read (possibly empty: no file), 0 = malformed or unreadable
int load(const char* path, std::map<std::string, Entry>* out) {
  FILE* f = fopen(path, "rb");
  if (!f) return errno == ENOENT ? 1 : 0;
  std::string text;
  char buf[4096];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
  const bool err = ferror(f) != 0;
  fclose(f);
  if (err) return 0;
  Reader r(text);
  return r.file(out) && r.ok ? 1 : 0;
}

void put_str(std::string* o, const std::string& s) {
  o->push_back('"');
  for (const char c : s) {
    if (c == '"' || c == '\\') {
      o->push_back('\\');
      o->push_back(c);
    } else if ((unsigned char)c < 0x20 || (unsigned char)c >= 0x80) {
      char u[8];
      snprintf(u, sizeof u, "\\u%04x", (unsigned)(unsigned char)c & 0x7Fu);  // no non-ASCII in signatures
      o->append(u);
    } else {
      o->push_back(c);
    }
  }
  o->push_back('"');
}

int save(const char* path, const std::map<std::string, Entry>& m) {
  std::string o = "{\"version\": 1, \"entries\": {";
  bool first = true;
  for (const auto& kv : m) {
    o += first ? "\n  " : ",\n  ";
    first = false;
    put_str(&o, kv.first);
    char b[64];
    snprintf(b, sizeof b, ": {\"method\": %d, \"choice\": %d, \"values\": [", kv.second.method, kv.second.choice);
    o += b;
    for (size_t k = 0; k < kv.second.values.size(); ++k) {
      snprintf(b, sizeof b, "%s%d", k ? ", " : "", kv.second.values[k]);
      o += b;
    }
    o += "], \"ms\": [";
    for (size_t k = 0; k < kv.second.ms.size(); ++k) {
      snprintf(b, sizeof b, "%s%.6g", k ? ", " : "", kv.second.ms[k]);
      o += b;
    }
    o += "]}";
  }
  o += "\n}}\n";
  static std::atomic<unsigned> seq{0};
  const std::string tmp = std::string(path) + ".tmp." + std::to_string((long)getpid()) + "." +
                          std::to_string(seq.fetch_add(1));
  FILE* f = fopen(tmp.c_str(), "wb");
  if (!f) return PTK_ERR_IO;
  const bool okw = fwrite(o.data(), 1, o.size(), f) == o.size();
  if (fclose(f) != 0 || !okw) {
    remove(tmp.c_str());
    return PTK_ERR_IO;
  }
  if (rename(tmp.c_str(), path) != 0) {
    remove(tmp.c_str());
    return PTK_ERR_IO;
  }
  return PTK_OK;
}

}  // namespace

extern "C" int ptk_tune_cache_lookup(const char* path, const char* signature, int32_t* found, int32_t* method,
                                     int32_t* choice) {
  if (!path || !signature || !found) return PTK_ERR_ARG;
  *found = 0;
  std::map<std::string, Entry> m;
  if (!load(path, &m)) return PTK_ERR_IO;
  const auto it = m.find(signature);
  if (it == m.end()) return PTK_OK;
  *found = 1;
  if (method) *method = it->second.method;
  if (choice) *choice = it->second.choice;
  return PTK_OK;
}

extern "C" int ptk_tune_cache_store(const char* path, const char* signature, int32_t method, int32_t choice,
                                    int32_t n, const int32_t* values, const float* ms) {
  if (!path || !signature || n < 0 || (n > 0 && (!values || !ms))) return PTK_ERR_ARG;
  std::map<std::string, Entry> m;
  if (!load(path, &m)) return PTK_ERR_IO;  // a malformed cache is left for its owner to inspect
  Entry e;
  e.method = method;
  e.choice = choice;
  for (int k = 0; k < n; ++k) {
    e.values.push_back(values[k]);
    e.ms.push_back(ms[k]);
  }
  m[signature] = e;
  return save(path, m);
}
