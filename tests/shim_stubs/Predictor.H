#pragma once
#include "gust_stubs.H"
