// Minimal JSON document reader for simulation_config.json and checkpoint
// metadata (objects, arrays, strings, numbers, true/false/null).
#pragma once

#include <cctype>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace tfiga::json {

struct Value {
	enum class Kind { Null, Bool, Number, String, Array, Object } kind = Kind::Null;
	bool boolean = false;
	double number = 0.0;
	std::string text;
	std::vector<Value> items;
	std::vector<std::pair<std::string, Value>> members;

	const Value* Find(const std::string& key) const
	{
		for (const auto& m : members) if (m.first == key) return &m.second;
		return nullptr;
	}
	const Value& At(const std::string& key, const std::string& context) const
	{
		const Value* v = Find(key);
		if (!v) throw std::runtime_error(context+" requires '"+key+"'");
		return *v;
	}
	double Number(const std::string& context) const
	{
		if (kind != Kind::Number) throw std::runtime_error(context+" must be a number");
		return number;
	}
	int Integer(const std::string& context) const
	{
		const double v = Number(context);
		if (v != (double)(long long)v) throw std::runtime_error(context+" must be an integer");
		return (int)v;
	}
	const std::string& String(const std::string& context) const
	{
		if (kind != Kind::String) throw std::runtime_error(context+" must be a string");
		return text;
	}
	const std::vector<Value>& Array(const std::string& context) const
	{
		if (kind != Kind::Array) throw std::runtime_error(context+" must be an array");
		return items;
	}
	bool IsObject() const { return kind == Kind::Object; }
};

class Parser {
public:
	explicit Parser(const std::string& text) : s_(text) {}
	Value Parse()
	{
		Value v = ParseValue();
		Skip();
		if (i_ != s_.size()) Error("trailing characters");
		return v;
	}

private:
	[[noreturn]] void Error(const std::string& what)
	{
		throw std::runtime_error("JSON parse error at offset "+std::to_string(i_)+": "+what);
	}
	void Skip() { while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_; }
	bool Eat(char c)
	{
		Skip();
		if (i_ < s_.size() && s_[i_] == c) { ++i_; return true; }
		return false;
	}
	void Expect(char c) { if (!Eat(c)) Error(std::string("expected '")+c+"'"); }
	Value ParseValue()
	{
		Skip();
		if (i_ >= s_.size()) Error("unexpected end");
		const char c = s_[i_];
		Value v;
		if (c == '{') {
			++i_;
			v.kind = Value::Kind::Object;
			if (Eat('}')) return v;
			do {
				Skip();
				std::string key = ParseString();
				Expect(':');
				Value member = ParseValue();
				// a repeated key is an error, with the message and byte position of the reference's
				// JSON reader (include/CaseConfig.hpp:124-142), which every case file goes through
				for (const auto& m : v.members)
					if (m.first == key)
						throw std::runtime_error("case_config.json: duplicate object key '"+key+"' at byte "
							+std::to_string(i_));
				v.members.emplace_back(std::move(key), std::move(member));
			} while (Eat(','));
			Expect('}');
		} else if (c == '[') {
			++i_;
			v.kind = Value::Kind::Array;
			if (Eat(']')) return v;
			do v.items.push_back(ParseValue()); while (Eat(','));
			Expect(']');
		} else if (c == '"') {
			v.kind = Value::Kind::String;
			v.text = ParseString();
		} else if (s_.compare(i_, 4, "true") == 0) {
			v.kind = Value::Kind::Bool; v.boolean = true; i_ += 4;
		} else if (s_.compare(i_, 5, "false") == 0) {
			v.kind = Value::Kind::Bool; i_ += 5;
		} else if (s_.compare(i_, 4, "null") == 0) {
			i_ += 4;
		} else {
			const char* begin = s_.c_str()+i_;
			char* end = nullptr;
			v.number = std::strtod(begin, &end);
			if (end == begin) Error("invalid value");
			v.kind = Value::Kind::Number;
			i_ += (size_t)(end-begin);
		}
		return v;
	}
	std::string ParseString()
	{
		if (i_ >= s_.size() || s_[i_] != '"') Error("expected string");
		++i_;
		std::string out;
		while (i_ < s_.size() && s_[i_] != '"') {
			char c = s_[i_++];
			if (c == '\\') {
				if (i_ >= s_.size()) Error("bad escape");
				const char e = s_[i_++];
				switch (e) {
				case 'n': c = '\n'; break;
				case 't': c = '\t'; break;
				case 'r': c = '\r'; break;
				case 'b': c = '\b'; break;
				case 'f': c = '\f'; break;
				case 'u': Error("unicode escapes are not supported");
				default: c = e;
				}
			}
			out.push_back(c);
		}
		if (i_ >= s_.size()) Error("unterminated string");
		++i_;
		return out;
	}
	const std::string& s_;
	size_t i_ = 0;
};

inline Value Parse(const std::string& text) { return Parser(text).Parse(); }

} // namespace tfiga::json
