// Stand-in for boost::gregorian as used by the reference's
// src/core/configuration.cpp (credit banner only: date -> "YYYY-Mon-DD").
#pragma once
#include <string>
#include <cstdio>
#include <cassert>   // boost/date_time brings this in transitively
namespace boost { namespace gregorian {
struct date {
	int y, m, d;
	date( int y_, int m_, int d_ ) : y(y_), m(m_), d(d_) {}
};
inline std::string to_simple_string( const date &dt ) {
	static const char *names[] = {"Jan","Feb","Mar","Apr","May","Jun","Jul","Aug","Sep","Oct","Nov","Dec"};
	char buf[32];
	std::snprintf(buf,sizeof(buf),"%04d-%s-%02d",dt.y,names[(dt.m+11)%12],dt.d);
	return buf;
}
}}
