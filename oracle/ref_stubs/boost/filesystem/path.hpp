/* Stand-in: boost::filesystem::path appears only in declarations on the paths compiled here. */
#pragma once
namespace boost { namespace filesystem { class path; } }
